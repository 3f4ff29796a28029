"""B200-native direct two-electron Fock build (J/K) for the polymer SCF code."""
