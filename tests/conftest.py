import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, 'tests', 'golden')


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA GPU (B200) and the built libpolymer_fock.so')
    config.addinivalue_line('markers', 'slow: takes more than ~10 s on the CPU')


@pytest.fixture(scope='session')
def reference_runs():
    with open(os.path.join(GOLDEN, 'reference_runs.json')) as fh:
        return json.load(fh)


def deck_of(run):
    from polymer_b200 import inputdeck
    return inputdeck.parse(inputdeck.deck_text(run['deck']['geometry'], run['deck']['keywords']))
