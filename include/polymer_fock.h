/*
 * polymer_fock.h -- C ABI of libpolymer_fock.so, the B200 direct J/K (Fock) build.
 *
 * Drop-in for SUBROUTINE FOURINDEX_ERI (src/pfourindexdirect.f90:1-814 of the
 * polymer code), which has no dummy arguments and communicates through Fortran
 * module globals.  pfe_args carries exactly the module state that subroutine
 * reads (src/pmodules.f90: BASISSET 74-93, INTEGRAL 111-160, STRUCTURE 35-45,
 * CONTROL DOPTN(12)/IOPTN(9), CONSTANTS MYID/NUMPROCS, FMT IGAMMA) and the two
 * outputs it overwrites, C_C and X_C (src/pmodules.f90:114-115).
 *
 * Every array is Fortran column-major with the reference's bounds; pointers are
 * borrowed for the duration of the call and never freed by the library.  All
 * entry points return 0 on success and a negative PFE_E* code on failure;
 * pfe_last_error() returns the message (the Fortran shim maps a non-zero code
 * to PABORT, src/pmain.f90:75-103).
 */
#ifndef POLYMER_FOCK_H
#define POLYMER_FOCK_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PFE_OK 0
#define PFE_EINVAL (-1)      /* malformed arguments (sizes, shell map, cutoffs) */
#define PFE_ECUDA (-2)       /* a CUDA runtime / cuBLAS call failed */
#define PFE_EUNSUPPORTED (-3)/* valid input outside what the kernels implement */
#define PFE_ERANGE (-4)      /* Boys order outside the IGAMMA table (reference: PABORT 'FMT CANNOT BE EVALUATED',
                                src/pfourindexdirect.f90:537-538).  Not reachable in this version: shells up to d
                                need orders <= 8 (9 for the gradient) of the table's 0..21, and higher shells are
                                refused with PFE_EUNSUPPORTED; the code is kept so that callers can map the abort. */
#define PFE_ENOMEM (-5)      /* device allocation failed */
#define PFE_ETIMEOUT (-6)    /* a bounded device wait gave up.  Not reachable in this version: no kernel waits on
                                another block, kernel or rank (work is handed out by atomic tickets), so there is
                                no device wait to bound. */
#define PFE_ENAN (-7)        /* non-finite density on input */

#define PFE_PREC_FP64 0      /* every quartet in FP64 (parity path) */
#define PFE_PREC_MIXED 1     /* molecules: quartets with Schwarz*|P|max below mixed_cutoff recur in FP32;
                                lattices: quartets whose ket image lies outside the CUTOFF1 box */

typedef struct pfe_args {
  int32_t npgs, ncgs, npshell;       /* NPGS, NCGS, NPSHELL (module BASISSET)            */
  int32_t lmax;                      /* BASIS_LMAX (3): P_SHELL is (npshell,0:lmax+1,...) */
  const int32_t *p_shell;            /* P_SHELL(npshell,0:lmax+1,0:lmax+1,0:lmax+1), 1-based, -1 = none */
  const int32_t *p_shell_ang;        /* P_SHELL_ANG(npshell)                              */
  const double *pgsx, *pgsy, *pgsz;  /* PGSX/Y/Z(npgs), bohr                              */
  const double *zt;                  /* ZT(npgs) exponents                                */
  const double *cc;                  /* CC(ncgs,npgs)                                     */
  const double *c2h;                 /* C2H(ncgs,ncgs,-(cel2x+cel1x):cel2x+cel1x); may be NULL if helix==0 */
  const double *s_p;                 /* S_P(npgs,npgs,-cel1x:cel1x,-cel1y:cel1y,-cel1z:cel1z) */
  const double *p_p;                 /* P_P, same layout as S_P                           */
  const double *p_p_helix;           /* P_P_HELIX(npgs,npgs,-cel2x:cel2x,-(cel2x+cel1x):cel2x+cel1x); NULL if helix==0 */
  const double *igamma;              /* IGAMMA(0:1700,0:27) (module FMT)                  */
  int32_t cel1[3], cel2[3];          /* CEL1X/Y/Z, CEL2X/Y/Z                              */
  int32_t reduced_cel1[3];           /* REDUCED_CEL1X/Y/Z (src/ponee.f90:359-409)         */
  double period[3];                  /* PERIODX/Y/Z, bohr                                 */
  double helix;                      /* HELIX, radians                                    */
  double inttol;                     /* DOPTN(12) (INTTOL)                                */
  int32_t print_level;               /* IOPTN(9) (PRINT); >=2 only affects the caller's dump */
  int32_t myid, numprocs;            /* MPI rank and size: this call computes rank myid's share;
                                        the caller sums C_C/X_C over ranks (MPI_ALLREDUCE)   */
  int32_t precision_mode;            /* PFE_PREC_FP64 or PFE_PREC_MIXED                   */
  double mixed_cutoff;               /* FP32 threshold on Schwarz(ij)*Schwarz(kl)*max|P|    */
} pfe_args;

/*
 * Replaces FOURINDEX_ERI (src/pfourindexdirect.f90:1-814), called each SCF
 * iteration from src/pselfconsistentfield.f90:42.  Host pointers in and out:
 * c_c and x_c are C_C/X_C(ncgs,ncgs,-cel1x:cel1x,-cel1y:cel1y,-cel1z:cel1z),
 * fully overwritten.  Static inputs (basis, S_P, IGAMMA, C2H, cutoffs) are
 * cached on the device under a hash of their contents, so only P_P/P_P_HELIX
 * are uploaded when they alone change between calls.
 */
int32_t pfe_fourindex_eri(const pfe_args *a, double *c_c, double *x_c);

/* Message of the most recent failure in this thread (NUL-terminated). Returns its length. */
int32_t pfe_last_error(char *buf, int32_t len);

/* ---- device-resident interface (no host round trip per SCF iteration) ---- */

typedef struct pfe_context pfe_context;

/* Create a context on CUDA device `device`; *out receives it. Builds nothing yet. */
int32_t pfe_context_create(int32_t device, pfe_context **out);
int32_t pfe_context_destroy(pfe_context *ctx);

/*
 * Upload static inputs and build the device pair lists / Schwarz bounds
 * (src/pfourindexdirect.f90:260-462 hoisted out of the SCF loop).  Only the
 * p_p / p_p_helix members of `a` are ignored.
 */
int32_t pfe_context_setup(pfe_context *ctx, const pfe_args *a);

/*
 * One Fock build with device pointers: d_p_p (and d_p_p_helix when helix != 0)
 * laid out as in pfe_args; d_c_c, d_x_c receive C_C/X_C.  `stream` is a
 * cudaStream_t (NULL = legacy default).  Lattices: asynchronous.  Molecules
 * whose CC gives every primitive at most one contracted function digest in
 * contracted space and read P_C off P_P; the call then synchronises the stream
 * to confirm P_P = CC^T P_C CC (the reference's P_P always is) and returns
 * PFE_EINVAL otherwise (inside a stream capture the confirmation is skipped).
 */
int32_t pfe_context_fock(pfe_context *ctx, const double *d_p_p, const double *d_p_p_helix,
                         double *d_c_c, double *d_x_c, void *stream);

/* Molecules: the same build from the contracted density d_p_c (ncgs x ncgs,
 * P_C of src/pdensitymatrix.f90, before DECONTRACT_DENSITYMATRIX), fully
 * asynchronous.  Replaces DECONTRACT_DENSITYMATRIX + FOURINDEX_ERI. */
int32_t pfe_context_fock_pc(pfe_context *ctx, const double *d_p_c, double *d_c_c, double *d_x_c, void *stream);

/* Runtime screening of molecular builds (no counterpart in the reference, whose
 * only screen is Schwarz(ij)*Schwarz(kl) < INTTOL).  With M = max|P| over the
 * density blocks a contracted shell quartet digests against: quartets with
 * Schwarz(ij)*Schwarz(kl)*M < density_tol are skipped (0 = off), and with
 * PFE_PREC_MIXED those with Schwarz(ij)*Schwarz(kl)*M < mixed_cutoff run the
 * recursion in FP32 (Boys function, geometry, contraction and J/K in FP64).
 * Meant for incremental builds from density differences.  Lattices and
 * helices: no density screening (PFE_EUNSUPPORTED); PFE_PREC_MIXED (with any
 * positive mixed_cutoff) runs the recursion of every quartet whose ket image
 * Q3 lies outside the CUTOFF1 box (the far cells) in FP32 and the near cells
 * in FP64 (Boys function, geometry and J/K accumulation stay FP64).  The same
 * holds for precision_mode/mixed_cutoff in pfe_args. */
int32_t pfe_context_set_screening(pfe_context *ctx, int32_t precision_mode, double mixed_cutoff,
                                  double density_tol);

/* Digest into primitive targets (then contract with CC on cuBLAS) even when
 * contracted targets are possible; takes effect at the next pfe_context_setup.
 * For callers whose P_P is not a decontracted density.  No counterpart in the
 * reference. */
int32_t pfe_context_primitive_targets(pfe_context *ctx, int32_t enable);

/* ---- batches of molecules (no counterpart in the reference) ----
 * Many molecules whose Fock builds run together: every instance is set up as
 * by pfe_context_setup, and one build runs one kernel launch per quartet class
 * (and pass) over every instance's work.  Densities and outputs are packed:
 * instance k's ncgs x ncgs column-major matrix starts at offset off[k] (in
 * doubles) of one device buffer; pfe_batch_offsets writes off[0..n] and returns n. */
typedef struct pfe_batch pfe_batch;
int32_t pfe_batch_create(int32_t device, pfe_batch **out);
/* Replaces any earlier set-up.  If one instance is refused (the status and
 * pfe_last_error say which), every instance is freed: until a set-up succeeds,
 * builds, screening, refresh and autotune return PFE_EINVAL, offsets and
 * schedule report none and the census is zero. */
int32_t pfe_batch_setup(pfe_batch *b, const pfe_args *instances, int32_t n);
int32_t pfe_batch_offsets(pfe_batch *b, int64_t *off);
/* pfe_context_set_screening applied to every instance. */
int32_t pfe_batch_set_screening(pfe_batch *b, int32_t precision_mode, double mixed_cutoff, double density_tol);
/* The same for instance k alone (0 <= k < n): instances of one build may use
 * different thresholds; an instance whose density difference is zero and whose
 * density_tol is positive skips all of its quartets. */
int32_t pfe_batch_set_instance_screening(pfe_batch *b, int32_t k, int32_t precision_mode, double mixed_cutoff,
                                         double density_tol);
int32_t pfe_batch_fock_pc(pfe_batch *b, const double *d_p_c, double *d_c_c, double *d_x_c, void *stream);
/* Graph capture: pfe_batch_fock_pc may be captured into a CUDA graph once its
 * launch records are current.  Every build uploads the records from a pinned
 * host copy, so a replay sees screening changed since the capture after this
 * call rewrites that copy for densities packed at d_p_c (the pointer captured);
 * call it with no replay in flight.  The kernels able to run FP32 are chosen at
 * capture: set a mixed cutoff on some instance before capturing if any replay
 * will use one. */
int32_t pfe_batch_refresh(pfe_batch *b, const double *d_p_c);
/* The schedule autotuner over a batch: times every execution variant of every
 * quartet class on the batch's densities d_p_c (packed) and keeps the fastest;
 * pfe_batch_schedule reports the classes (cls, chosen variant, tuned_ms,
 * quartets, flops; ms = 0) and returns their number. */
int32_t pfe_batch_autotune(pfe_batch *b, const double *d_p_c, void *stream);
int32_t pfe_batch_destroy(pfe_batch *b);

/* Screened-quartet census and algorithmic FLOPs of the last setup (per Fock build). */
typedef struct pfe_census {
  double quartets;          /* screened primitive-shell quartets computed per build   */
  double quartets_ref;      /* lattices: the same work counted the reference's way (no
                               symmetry); molecules: 0 (not counted; the reference's
                               loop evaluates up to 8 orderings of each quartet)     */
  double flops;             /* FP64/FP32 recursion + digestion flops per build        */
  double quartets_fp32;     /* quartets routed to FP32 recursion (mixed mode)          */
  int64_t pairs;            /* significant primitive-shell pairs kept                 */
  int32_t kernel_launches;  /* kernels launched by one pfe_context_fock call          */
} pfe_census;
int32_t pfe_context_census(pfe_context *ctx, pfe_census *out);
/* The same summed over a batch's instances (kernel_launches: one batched build). */
int32_t pfe_batch_census(pfe_batch *b, pfe_census *out);

/* Per-kernel timing of pfe_context_fock (diagnostics; no counterpart in the
 * reference).  With profiling on, every quartet-class launch is bracketed by
 * CUDA events on the caller's stream; pfe_context_kernel_stats() (after the
 * stream is synchronised) returns, per launch of the last Fock build, the class
 * code 1000*LA+100*LB+10*LC+LD, the milliseconds, the screened quartets and the
 * algorithmic flops.  Returns the number of launches written. */
int32_t pfe_context_profile(pfe_context *ctx, int32_t enable);
typedef struct pfe_kernel_stat {
  int32_t cls;
  int32_t variant;    /* 0 straight-line thread/quartet, 1 warp/quartet, 2 block/quartet,
                         3 warp/quartet with per-lane Boys and geometry, kept outputs only */
  float ms;
  float tuned_ms[4];  /* autotuner timing of each variant, 0 where not run */
  double quartets;
  double flops;
  int32_t grid_mult;  /* straight-line variant: blocks per SM of its persistent grid */
  int32_t pad_;
} pfe_kernel_stat;
int32_t pfe_context_kernel_stats(pfe_context *ctx, pfe_kernel_stat *out, int32_t cap);
/* A batch's quartet classes and their schedule (see pfe_batch_autotune). */
int32_t pfe_batch_schedule(pfe_batch *b, pfe_kernel_stat *out, int32_t cap);

/* Schedule autotuning (no counterpart in the reference): time every execution
 * variant of every quartet class on this context's screened work lists with the
 * device density d_p_p, keep the fastest for later builds.  Synchronous.  The
 * host entry point pfe_fourindex_eri runs it on its first call after a set-up. */
int32_t pfe_context_autotune(pfe_context *ctx, const double *d_p_p, const double *d_p_p_helix, void *stream);

/* Force execution variant v (0..3 as in pfe_kernel_stat) on every quartet
 * class that has it; the others keep theirs (diagnostics and tests). */
int32_t pfe_context_force_variant(pfe_context *ctx, int32_t variant);

/* Replaces the molecular branch of FOURINDEX_ERI_GRADIENT
 * (src/pfourindexgradient.f90:1-1478), which adds the two-electron part of the
 * nuclear gradient to FORCEX/Y/Z(NATOM) (module GRADIENT).  Same argument
 * block as pfe_fourindex_eri (P_P the density; molecules only: a lattice or
 * helix returns PFE_EUNSUPPORTED) plus PGS_ATOM(npgs) (1-based atom of every
 * primitive) and natom.  grad_j and grad_k (natom x 3, column-major: the x
 * derivatives of all atoms, then y, then z) are overwritten with
 *   grad_j = d/dR [ 1/2 sum (ij|kl) P_ij P_kl ],  grad_k = d/dR [ -1/4 sum (ij|kl) P_ik P_jl ]
 * at fixed P; the reference's two-electron force is grad_j + HFX * grad_k
 * (HFX = DOPTN(19)).  Host pointers; synchronous. */
int32_t pfe_fourindex_eri_gradient(const pfe_args *a, const int32_t *pgs_atom, int32_t natom, double *grad_j,
                                   double *grad_k);

/* Measured FP64 FMA-pipe throughput of `device` in TFLOP/s (a dependent-chain
 * free DFMA loop over all SMs; diagnostics for the roofline denominator). */
int32_t pfe_measure_fp64_peak(int32_t device, double *tflops);

/* ---- caller-side set-up integrals (outside FOURINDEX_ERI) ----
 * The Fortran caller computes these before the SCF (src/psinglepoint.f90:184,212);
 * they are provided on the device so a host driver needs no CPU integral code. */
typedef struct pfe_onee_args {
  int32_t npgs, npshell, natom;
  const int32_t *p_shell, *p_shell_ang, *pgs_atom; /* as in pfe_args; PGS_ATOM(npgs) 1-based */
  const double *pgsx, *pgsy, *pgsz, *zt;
  const int32_t *iatom;                           /* IATOM(natom) nuclear charges          */
  const double *atomx, *atomy, *atomz;            /* ATOMX/Y/Z(natom), bohr                 */
  int32_t cel1[3], cel2[3];
  double period[3], helix;
  const double *igamma;                           /* IGAMMA(0:1700,0:27)                    */
} pfe_onee_args;

/* OVERLAP_KINETIC(0) (src/ponee.f90:1-160): S_P and T_P(npgs,npgs,cells1), host out. */
int32_t pfe_overlap_kinetic(const pfe_onee_args *a, double *s_p, double *t_p);
/* NUCLEAR_ATTRACTION(0) (src/ponee.f90:418-603): N_P(npgs,npgs,cells1), host out. */
int32_t pfe_nuclear_attraction(const pfe_onee_args *a, double *n_p);

/* No counterpart in the reference.  pfe_overlap_kinetic without any device
 * allocation: for callers that may not allocate device memory while running
 * (a fixed memory budget, an allocator that owns the device).  Its device data
 * live in one 16 MiB array compiled into the library, so the inputs and
 * 2*npgs*npgs*cells1 results must fit there (a 976-primitive molecule does);
 * larger inputs return PFE_EINVAL with the size needed.  The first call on a
 * device does the set-up (module load and symbol lookup on that device) and
 * should come before any stream capture; the address found then is kept for
 * the life of the process, so a cudaDeviceReset between calls is not
 * supported.  Calls share the one buffer per device, so they are serialised
 * by a lock; host buffers as pfe_overlap_kinetic.  P_SHELL entries of every
 * component a shell reaches must name primitives 1..npgs (else PFE_EINVAL,
 * checked before any device work). */
int32_t pfe_overlap_kinetic_noalloc(const pfe_onee_args *a, double *s_p, double *t_p);

/* Library version string. */
const char *pfe_version(void);

/* Testing aid, no reference counterpart: the `after`-th device allocation that a
 * context or batch set-up asks for from now on (0: the next one) fails as if the
 * device were out of memory, so that callers can exercise their PFE_ENOMEM
 * paths; the failing call returns PFE_ENOMEM and leaves its context or batch not
 * set up (a later set-up starts afresh).  Negative `after`: no injection (the
 * default).  Process-wide; nothing is attempted on the device. */
int32_t pfe_debug_fail_allocation(int32_t after);

#ifdef __cplusplus
}
#endif

#endif /* POLYMER_FOCK_H */
