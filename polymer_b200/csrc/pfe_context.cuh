// Device-side state of one Fock-build context (struct pfe_context of the C ABI).
#pragma once

#include <atomic>

#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "pfe_common.cuh"

namespace pfe {

// Allocation-failure injection for tests of the error paths: the n-th device
// allocation a context or batch asks for from now on fails as out of memory
// (pfe_debug_fail_allocation); negative: never.  Nothing reaches the GPU: the
// allocation is simply not attempted.
inline std::atomic<long long> g_fail_alloc_after{-1};

inline cudaError_t injected_alloc_failure() {
  long long v = g_fail_alloc_after.load();
  while (v >= 0)
    if (g_fail_alloc_after.compare_exchange_weak(v, v - 1)) return v == 0 ? cudaErrorMemoryAllocation : cudaSuccess;
  return cudaSuccess;
}


// Primitive-shell table, struct of arrays (n shells).
struct DevShells {
  int n;
  double *x, *y, *z, *zeta;
  int* L;
  int* prim;  // n * MAXCOMP, 0-based primitive of each cumulative component (-1 ghost/absent)
};

// Shell-pair records, struct of arrays; sorted by class and bound after setup.
struct PairArrays {
  double* P[3];
  double* PA[3];
  double* AB[3];
  double* zeta;
  double* S;        // S_P of the two s components (the reference's OV / C1 factor)
  double* schwarz;  // the reference's IJIJ/KLKL bound
  int* si;
  int* sj;
  unsigned char* cls;
  unsigned long long* key;
  int* gid;         // contracted block pair (molecules)
  double* gmax;     // largest bound in the pair's block-pair group (molecules)
};

// One launch of the quartet kernel: a (bra class, ket class) pair and its chunks.
struct ClassLaunch {
  int cb, ck;
  int nchunks_host;
  int* d_nchunks;
  int4* chunks;  // (bra pair, first ket, end ket, 0)
  double quartets;
  // execution variant: 0 = straight-line thread per quartet, 1 = warp per
  // quartet on the op table, 2 = block per quartet on the op table, 3 = warp
  // per quartet on the op table with per-lane Boys/geometry and only the
  // outputs that carry a coefficient (pfe_mol_wide.cu)
  int variant;
  bool has_straight, has_table;
  const unsigned short* ops;
  const int* levels;
  const unsigned short* out;
  int nlevels, nout, nslots;
  const unsigned short* ops_p;   // pure-bra table (see OpTableDev), or null
  const int* levels_p;
  const unsigned short* out_p;
  int nlevels_p;
  const unsigned short* ops_p2;  // pure bra and pure ket table, or null
  const int* levels_p2;
  const unsigned short* out_p2;
  int nlevels_p2;
  int wpb, per_warp;         // warps per block and doubles per warp (variant 1)
  size_t smem_big, smem_warp;
  float tuned_ms[4];         // autotuner timings per variant (0 = not run)
  double* xg;                // block variant: per-block X scratch in global memory, or null
  int nslots_p, nslots_p2;   // slots of the pure-bra and bra-and-ket tables (0: none)
  // variant 3 (warp per primitive quartet, kept outputs only): per-warp shared
  // memory in doubles, of which wide_vmax op-table slots and wide_xmax outputs
  bool has_wide;
  int wide_wpb, wide_per_warp, wide_vmax, wide_xmax;
  size_t smem_wide;
  int* queue;                // device work queue: one chunk counter per launch (pass), zeroed before each
  unsigned int* cost;        // screened primitive quartets per chunk (chunks are sorted by it, descending)
  int npass;                 // register passes of the straight-line variant
  int npass_live;            // of which launched: the others keep no component with a coefficient
  int gmul = 32;             // straight-line variant: persistent grid of up to gmul blocks per SM
};

}  // namespace pfe

// The opaque handle of the C ABI.
struct pfe_context {
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  // the interpreter classes' launches run on `side`, beside the straight-line
  // classes on the caller's stream (forked and joined with the two events)
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  cublasHandle_t blas = nullptr;
  bool ready = false;
  uint64_t key = 0;
  bool molecular = true;
  int npgs = 0, ncgs = 0, npshell = 0, ncell1 = 1;
  int cel1[3] = {0, 0, 0}, cel2[3] = {0, 0, 0}, rc1[3] = {0, 0, 0};
  double period[3] = {0, 0, 0};
  double helix = 0.0;
  double inttol = 0.0;
  int myid = 0, numprocs = 1;
  int precision = 0;
  double mixed_cutoff = 0.0;

  // device data
  pfe::DevShells shells{};
  double* d_sss = nullptr;   // S_P(head I, head J, cell) for shell heads, [cell][J][I]
  double* d_boys = nullptr;
  double* d_maxc = nullptr;  // max_i |CC(i, p)| per primitive
  double* d_cc = nullptr;    // CC (ncgs x npgs, column-major)
  double* d_c2h = nullptr;
  double* d_jp = nullptr;
  double* d_kp = nullptr;
  // digestion targets: contracted functions when every primitive feeds at most
  // one contracted row of CC (the reference's READ3 bases), else primitives
  bool contracted = false;
  int nt = 0;                // target dimension (ncgs or npgs)
  int* d_tidx = nullptr;     // primitive -> target row, -1 when it has no coefficient
  double* d_tcoef = nullptr; // primitive -> coefficient (CC entry, or 1)
  double* d_scoef = nullptr; // shell x component -> coefficient of its primitive (tcoef)
  int* d_stidx = nullptr;    // shell x component -> target row of its primitive (tidx)
  int* d_blk = nullptr;      // shell -> contracted block id
  // per angular momentum L of a shell: the most components with a target row
  // one shell of that L has, and whether some shell of that L has a target on
  // a component below L (a cumulative sp/spd shell, not a pure p/d one)
  int kept_max[3] = {1, 4, 10};
  bool lower_kept[3] = {false, true, true};
  int nblk = 0;
  bool force_primitive = false;  // set before set-up: primitive targets even when CC allows contracted ones
  int* d_rep = nullptr;      // target -> representative primitive (largest |coefficient|)
  double* d_repc = nullptr;  // its coefficient
  double* d_pt = nullptr;    // density in target space (nt x nt): P_C read off P_P, or P_P
  unsigned int* d_flag = nullptr;  // set when P_P is not the decontraction of a contracted density
  // groups: runs of pairs of one contracted block pair (molecules)
  void* d_prec = nullptr;    // the sorted pairs as 128-byte records (PairRec)
  int ngroups = 0;
  int* d_gr_start = nullptr;
  int* d_gr_n = nullptr;
  double* d_gr_max = nullptr;
  int* d_bk_list = nullptr;  // group ids ordered by (class, size bucket, group)
  // density-dependent screening of molecular builds (no counterpart in the reference, which
  // screens by the Schwarz bounds alone): skip quartets with bound * max|P| < dtol, and run
  // the recursion in FP32 where bound * max|P| < mcut; max|P| per pair of contracted blocks
  double dtol = 0.0, mcut = 0.0;
  int* d_tblk = nullptr;     // target -> block (-1: none)
  double* d_bmax = nullptr;  // nblk x nblk block maxima of |P_T| of the last build
  unsigned long long* d_n32 = nullptr;  // quartets of the last build run in FP32
  double* d_w1 = nullptr;
  double* d_w2 = nullptr;
  pfe::PairArrays pairs{};
  long long npairs = 0;
  int class_off[8] = {0}, class_n[8] = {0};
  pfe::ClassLaunch launches[64];
  int nlaunch = 0;
  int* d_queue = nullptr;    // 64 chunk counters per class launch (the work queues of launches[])
  double census_quartets = 0.0, census_flops = 0.0, census_ref = 0.0, census_fp32 = 0.0;

  // host-path staging (pfe_fourindex_eri)
  double* d_pp = nullptr;
  double* d_pph = nullptr;
  double* d_out_c = nullptr;
  double* d_out_x = nullptr;
  size_t pp_bytes = 0, pph_bytes = 0, out_bytes = 0;

  // lattice path state lives in pfe_lattice.cu
  void* lattice = nullptr;

  // per-launch timing (pfe_context_profile)
  bool profile = false;
  bool tuned = false;
  cudaEvent_t ev[130] = {};
  int nev = 0;
  int ev_cls[64] = {0};
  int ev_variant[64] = {0};
  float ev_tuned[64][4] = {};
  double ev_quartets[64] = {0}, ev_flops[64] = {0};
  int ev_gmul[64] = {0};
  int nprof = 0;

  std::vector<void*> owned;    // freed on reset/destroy
  std::vector<void*> pending;  // scratch freed at the end of setup

  cudaError_t alloc(void** p, size_t bytes) {
    if (cudaError_t f = pfe::injected_alloc_failure()) return f;
    cudaError_t e = cudaMalloc(p, bytes ? bytes : 16);
    if (e == cudaSuccess) owned.push_back(*p);
    return e;
  }
  void free_now(void* p) {
    if (!p) return;
    for (size_t i = 0; i < owned.size(); ++i)
      if (owned[i] == p) {
        owned.erase(owned.begin() + i);
        break;
      }
    cudaFree(p);
  }
  void free_later(void* p) { pending.push_back(p); }
  void free_pending() {
    for (void* p : pending) free_now(p);
    pending.clear();
  }
  void release_all() {
    for (void* p : owned) cudaFree(p);
    owned.clear();
    pending.clear();
  }
};

// Many molecules whose Fock builds run together (struct pfe_batch of the C ABI):
// every instance has its own context (set-up, pairs, chunks); the batch joins
// their chunk lists per quartet class, each chunk tagged with its instance, so
// one launch per class (and pass) covers every instance.
struct pfe_batch {
  int device = 0;
  std::vector<pfe_context*> inst;
  std::vector<long long> off;       // packed offsets (doubles) of the ncgs x ncgs matrices, n+1
  pfe::ClassLaunch launches[64];    // joined chunk lists; ops/tables of the first instance with the class
  int nlaunch = 0;
  int* d_queue = nullptr;           // the joined launches' work queues (64 counters each)
  long long* d_off = nullptr;       // off[] on the device (the batched symmetrisation)
  bool all_contracted = false;      // every instance digests in contracted space
  void* d_insts = nullptr;          // the instances' launch records (MolLaunch) on the device
  void* h_insts = nullptr;          // ... and their pinned host copy, uploaded by every build (so a
                                    // captured graph re-reads it at each replay)
  cudaEvent_t ev_insts = nullptr;   // the last upload of h_insts
  bool ev_pending = false;
  const double* insts_for = nullptr;  // density the records point at (null: rewrite them)
  bool mixed = false;               // FP32-capable kernels (sticky once any instance asked for them)
  bool ready = false;               // set by a pfe_batch_setup that succeeded
  std::vector<void*> owned;
  cudaError_t alloc(void** p, size_t bytes) {
    if (cudaError_t f = pfe::injected_alloc_failure()) return f;
    cudaError_t e = cudaMalloc(p, bytes ? bytes : 16);
    if (e == cudaSuccess) owned.push_back(*p);
    return e;
  }
  void release_all() {
    for (void* p : owned) cudaFree(p);
    owned.clear();
    if (h_insts) cudaFreeHost(h_insts);
    h_insts = nullptr;
    if (ev_insts) cudaEventDestroy(ev_insts);
    ev_insts = nullptr;
    ev_pending = false;
    d_insts = nullptr;
    insts_for = nullptr;
    nlaunch = 0;   // the launches pointed into the memory freed above
    ready = false;
  }
};

namespace pfe {
// The context's cuBLAS handle, created on first use: molecules with contracted
// targets never call cuBLAS, and a batch holds hundreds of contexts.
inline bool ensure_blas(pfe_context* ctx) {
  if (ctx->blas) return true;
  if (cublasCreate(&ctx->blas) != CUBLAS_STATUS_SUCCESS) {
    ctx->blas = nullptr;
    return false;
  }
  return true;
}
int batch_setup(pfe_batch* b);
int batch_fock_pc(pfe_batch* b, const double* d_pc, double* d_cc, double* d_xc, cudaStream_t s);
int batch_refresh(pfe_batch* b, const double* d_pc);
int batch_autotune(pfe_batch* b, const double* d_pc, cudaStream_t s);
int alloc_pairs(pfe_context* ctx, PairArrays* pa, long long n);
void free_pairs(pfe_context* ctx, PairArrays* pa);
void launch_symmetrize(const double* a, double* out, int n, int ncell, cudaStream_t s);
void launch_select_class(const unsigned char* cls, int want, int* list, int* count, long long n, cudaStream_t s);
int upload_constants(int device);
int molecular_setup(pfe_context* ctx, const pfe_args* a);
int molecular_fock(pfe_context* ctx, const double* d_pp, double* d_cc, double* d_xc, cudaStream_t s);
int contract_outputs(pfe_context* ctx, const double* jp, const double* kp, double* d_cc, double* d_xc,
                     bool symmetrize, int ncell, cudaStream_t s);
int autotune(pfe_context* ctx, const double* d_pp, cudaStream_t s);
int molecular_density_ok(pfe_context* ctx, cudaStream_t s, bool* ok);
int molecular_fock_pc(pfe_context* ctx, const double* d_pc, double* d_cc, double* d_xc, cudaStream_t s);
struct OpTableDev;
const struct OpTableHost* host_optable(int cb, int ck);
const struct OpTableHost* host_optable_pure(int cb, int ck);
const struct OpTableHost* host_optable_pure2(int cb, int ck);
int upload_optable(pfe_context* ctx, const struct OpTableHost* h, OpTableDev* d);
double class_flops(int cb, int ck);
int lattice_setup(pfe_context* ctx, const pfe_args* a);
int lattice_fock(pfe_context* ctx, const double* d_pp, const double* d_pph, double* d_cc, double* d_xc,
                 cudaStream_t s);
void lattice_release(pfe_context* ctx);
void lattice_force_interpreter(pfe_context* ctx, bool on);
int lattice_class_launches(pfe_context* ctx);
int molecular_gradient_pp(pfe_context* ctx, const double* d_pp, const int* d_satom, int natom, double* d_gj,
                          double* d_gk, cudaStream_t s);
const char* last_error_cstr();
int measure_fp64_peak(int device, double* tflops);
}  // namespace pfe
