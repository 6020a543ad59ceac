/*
 * cqgpu: B200 (sm_100a) direct-SCF two-electron engine -- C ABI.
 *
 * Drop-in for ChronusQ's AOIntegrals direct two-electron contraction.  Every matrix is
 * real FP64, nbf x nbf, column-major with leading dimension `ld` (>= nbf), basis
 * functions ordered as the reference orders them: atom order, then the .gbs shell
 * order (SP split S then P), then components (Cartesian x^l, x^(l-1)y, x^(l-1)z, ...;
 * real solid harmonics m=-l..l for pure shells).  Results ACCUMULATE into AX (AX +=),
 * as the reference does; callers zero AX first when they want G alone.
 *
 * Pointers are host pointers when `on_device` is 0 (the call copies in and out on
 * `stream`, and returns after the copy-out has completed) and device pointers of the
 * context's device when `on_device` is 1 (the call only enqueues work on `stream`).
 * `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 *
 * Errors are returned as cqg_status; nothing aborts or traps on the device.
 * A context is not safe for concurrent use from several threads.
 */
#ifndef CQGPU_H
#define CQGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  CQG_OK = 0,
  CQG_ERR_BAD_ARG = 1,       /* reference: assert on list sizes (aointegrals_contract.h:31-33) */
  CQG_ERR_OOM = 2,           /* reference: std::bad_alloc from CQMemManager (memory.h:65-88) */
  CQG_ERR_CUDA = 3,          /* a CUDA runtime call failed */
  CQG_ERR_TIMEOUT = 4,       /* a bounded device wait gave up */
  CQG_ERR_NONFINITE = 5,     /* NaN/Inf found in an input density */
  CQG_ERR_STATE = 6,         /* call order violated (e.g. contraction before basis) */
  CQG_ERR_UNSUPPORTED = 7    /* outside what this engine implements (see cqg_last_error) */
} cqg_status;

/* ERI_CONTRACTION_TYPE (include/aointegrals.h:468-472) */
enum { CQG_COULOMB = 0, CQG_EXCHANGE = 1 };

/* precision policy of the quartet evaluation */
enum {
  CQG_PREC_FP64 = 0,         /* every quartet in FP64 (the reference's arithmetic) */
  CQG_PREC_MIXED = 1         /* quartets whose density-weighted Schwarz bound (the screen's
                                max block norm * Q_ab * Q_cd) is below the FP32 cutoff are
                                evaluated in FP32, accumulated in FP64 */
};

typedef struct cqg_ctx cqg_ctx;

/* statistics of the last contraction on a context */
typedef struct {
  long long quartets;              /* screened unique shell quartets (the unit of work) */
  long long quartets_fp32;         /* of which evaluated in FP32 (mixed policy) */
  long long prim_quartets;         /* primitive quartets evaluated */
  double model_flops;              /* MD-v1 model FLOPs of the screened quartets */
  double model_flops_fp32;         /* of which in FP32 quartets */
  double ms_screen;                /* device time of screening + list build (ms) */
  double ms_eri;                   /* device time of ERI + digest kernels (ms) */
  double ms_total;                 /* device time of the whole call (ms) */
  long long launches;              /* kernels of this library launched by the call */
  long long chunks;                /* quartet-list chunks the call was processed in */
  long long class_quartets[55];    /* per quartet class (index: see cqg_class_name) */
  double class_ms[55];             /* device time per class kernel (ms), if timing on */
  double ms_fused;                 /* device time of the class-fused kernel (ms), if timing on */
  int fused_tier;                  /* 0: per-class launches; 1, 2: class-fused tier used */
  long long list_entries;          /* quartet-list entries (a sibling-group entry holds up to 16
                                      quartets; without siblings one entry per quartet) */
  long long sibling_classes;       /* bit k set: class k's lists held sibling-group entries */
} cqg_stats;

/* Library / context lifetime. */
const char *cqg_version(void);
const char *cqg_status_string(cqg_status s);
cqg_status cqg_create(cqg_ctx **ctx, int device);
cqg_status cqg_destroy(cqg_ctx *ctx);
const char *cqg_last_error(const cqg_ctx *ctx);

/* Basis upload (replaces BasisSet::shells_ + mapSh2Bf, include/basisset.h;
 * src/basisset/basisset_map.cpp:29-40).  Per shell: angular momentum L, pure flag
 * (1 = spherical; the engine requires pure == (L > 1), the reference default at
 * src/basisset/basisset_read.cpp:250-251), primitive count; alpha/coef are the
 * concatenated exponents and NORMALISED contraction coefficients (as held by a
 * libint2::Shell after renormShells, src/basisset/basisset_misc.cpp:95-111);
 * centers is nshell x 3 in bohr.  Computes the Schwarz bounds on the device
 * (AOIntegrals::computeSchwartz, src/aointegrals/aointegrals_builders.cpp:469-517). */
cqg_status cqg_set_basis(cqg_ctx *ctx, int nshell, const int *L, const int *pure,
                         const int *nprim, const double *alpha, const double *coef,
                         const double *centers);

/* AOIntegrals::thresholdSchwartz_ (include/aointegrals.h:334; default 1e-14). */
cqg_status cqg_set_threshold(cqg_ctx *ctx, double thresh);

/* Precision policy; `fp32_cutoff` is the density-weighted bound below which a quartet runs
 * in FP32 under CQG_PREC_MIXED. */
cqg_status cqg_set_precision(cqg_ctx *ctx, int policy, double fp32_cutoff);

/* Copy the nshell x nshell Schwarz matrix (column-major) to host memory. */
cqg_status cqg_get_schwarz(cqg_ctx *ctx, double *Q);
cqg_status cqg_get_sizes(cqg_ctx *ctx, int *nshell, int *nbasis, int *maxl);

/* AOIntegrals::newTwoEContractDirect (include/aointegrals/aointegrals_contract.h:24-194,
 * declared include/aointegrals.h:474-480) for real matrices:
 *   for i < nmat:  AX[i] += 0.5 * scale[i] * G_i[X[i]]
 * with G = 4 J[X] for types[i] == CQG_COULOMB and G = 4 K[X] for CQG_EXCHANGE (so
 * AX += scale * 2J or scale * 2K), J_mn = sum (mn|ls) X_ls, K_mn = sum (ml|ns) X_ls,
 * over the unique shell quartets that pass the reference's density-weighted Schwarz
 * screen.  X must be symmetric (the engine checks and returns CQG_ERR_UNSUPPORTED
 * otherwise).  Entries sharing the same X and AX pointers are fused into one pass. */
cqg_status cqg_twoe_contract_direct(cqg_ctx *ctx, int nmat, const double *const *X,
                                    double *const *AX, const int *types, const double *scale,
                                    int ld, int on_device, void *stream);

/* SingleSlater<double>::formPT (include/singleslater/singleslater_fock.h:31-93): zeroes
 * PTs (and PTz) and builds  RHF: PTs = 2J[Ps] + 2 xHF K[Ps]
 *                           UHF: additionally PTz = 2 xHF K[Pz]
 * (xHF = -0.5 for Hartree-Fock, include/singleslater.h:455).  Pz/PTz NULL for RHF. */
cqg_status cqg_form_pt(cqg_ctx *ctx, int is_rhf, double xHF, const double *Ps,
                       const double *Pz, double *PTs, double *PTz, int ld, int on_device,
                       void *stream);

/* One-electron integrals on the device: overlap S, kinetic T and nuclear attraction V
 * of `ncharge` point charges Z at R (ncharge x 3, bohr), each nbf x nbf (leading dim
 * `ld`), in the same basis-function order.  Replaces AOIntegrals::computeAOOneE's
 * OneEDriver calls (src/aointegrals/aointegrals_builders.cpp:27-133, 337-467). */
cqg_status cqg_one_e(cqg_ctx *ctx, int ncharge, const double *Z, const double *R, double *S,
                     double *T, double *V, int ld, int on_device, void *stream);

/* Electric dipole integrals <mu| r_k - origin_k |nu>, k = x, y, z, of a single-molecule
 * context: D holds the three nbf x nbf matrices (column-major, leading dimension ld) at D,
 * D + ld * nbf and D + 2 * ld * nbf, host or device memory as `on_device` says.  Replaces
 * the first electric multipole integrals of AOIntegrals::computeAOOneE
 * (AOIntegrals::elecDipole_, split per component in AOIntegrals::breakUpMultipole,
 * src/aointegrals/aointegrals_builders.cpp:640-650), which SingleSlater adds to the Fock
 * matrix in a static field (AOIntegrals::subElecDipole, include/aointegrals.h:505-510). */
cqg_status cqg_dipole(cqg_ctx *ctx, const double *origin, double *D, int ld, int on_device, void *stream);

/* cqg_one_e without any allocation: the same integrals and kernel as cqg_one_e with device
 * S, T, V (leading dimension ld), but the point-charge table is held in a fixed
 * module-scope device array of CQG_ONE_E_NOALLOC_MAX_CHARGES entries (4 doubles each,
 * 128 KiB) instead of context scratch, so the call makes no cudaMalloc/cudaFree and calls
 * no allocating library.  Z and R may be host or device pointers; work is enqueued on
 * `stream`, nothing is synchronised: pinned or device Z/R are read when the stream reaches
 * the copy, so keep them alive until then; under stream capture pass device or pinned Z/R
 * (a pageable host copy cannot be captured).  ncharge > CQG_ONE_E_NOALLOC_MAX_CHARGES and
 * ld < nbf return CQG_ERR_BAD_ARG (cqg_last_error says why) before anything is written.
 * Nothing has to start at zero: the table is written in full for the entries read and
 * every element of the nbf x nbf blocks of S, T, V is written (rows nbf..ld-1 are not).
 * The first call on a context resolves the array's device address (cudaGetSymbolAddress,
 * with the context's device current) and keeps it in the context; make that first call
 * before any stream capture.  The array is shared by every context on a device: calls that
 * overlap (other streams, threads or contexts on the same device) race on it and must be
 * serialised by the caller.
 * This entry point has no counterpart in the reference. */
#define CQG_ONE_E_NOALLOC_MAX_CHARGES 4096
cqg_status cqg_one_e_noalloc(cqg_ctx *ctx, int ncharge, const double *Z, const double *R,
                             double *S, double *T, double *V, int ld, void *stream);

/* ---- Batches: many independent molecules of uneven size in one context ----
 * cqg_set_basis_batch takes the shells of all molecules concatenated (molecule m has
 * nshell_per_mol[m] shells).  Matrices of a batch live on the device, packed: molecule m's
 * nbf_m x nbf_m matrix (leading dimension nbf_m) starts at offset_per_mol[m] (elements)
 * of one array (cqg_get_batch_layout).  One batched contraction evaluates the quartets of
 * every active molecule in the same class kernels (one work list per quartet class). */
cqg_status cqg_set_basis_batch(cqg_ctx *ctx, int nmol, const int *nshell_per_mol, const int *L,
                               const int *pure, const int *nprim, const double *alpha,
                               const double *coef, const double *centers);
cqg_status cqg_get_batch_layout(cqg_ctx *ctx, int *nbf_per_mol, long long *offset_per_mol,
                                long long *packed);
/* newTwoEContractDirect for every molecule m with active[m] != 0 (NULL: all), device
 * pointers to packed matrices; same list semantics as cqg_twoe_contract_direct. */
cqg_status cqg_twoe_contract_direct_batch(cqg_ctx *ctx, int nmat, const double *const *X,
                                          double *const *AX, const int *types,
                                          const double *scale, const unsigned char *active,
                                          void *stream);
/* One-electron integrals of every molecule of a batch (charges concatenated per molecule,
 * ncharge_per_mol[m] of them), into packed device S, T, V. */
cqg_status cqg_one_e_batch(cqg_ctx *ctx, const int *ncharge_per_mol, const double *Z,
                           const double *R, double *S, double *T, double *V, void *stream);

/* ---- CUDA graphs and launch shapes ----
 * cqg_set_graph_mode(ctx, capacity, max_groups): capacity > 0 makes device-pointer
 * contractions free of host synchronisation so they can be captured in a CUDA graph and
 * replayed (one graph per SCF iteration shape).  The quartet list holds at most `capacity`
 * quartets and up to `max_groups` distinct (X, AX) pairs are allowed per call; after a
 * replay, cqg_graph_status reports the screened quartet count and whether the capacity
 * overflowed (the result is then incomplete and must be recomputed with a larger
 * capacity) or the input was non-finite / asymmetric.  capacity = 0 restores the default.
 * Per-class statistics are not collected in graph mode. */
cqg_status cqg_set_graph_mode(cqg_ctx *ctx, long long capacity, int max_groups);
cqg_status cqg_graph_status(cqg_ctx *ctx, long long *quartets, int *overflow, int *nonfinite,
                            int *asymmetric);
/* Autotuner: the next (non-graph, single-chunk) contraction times every candidate launch
 * shape of each class work list (persistent CTAs per SM; warps per CTA for the
 * warp-cooperative classes; quartets claimed per warp from the list's work queue) and keeps
 * the fastest for later calls.  The shapes are read
 * back with cqg_get_launch_shapes (cqg_schedule_lists() entries: FP64 lists then FP32 lists;
 * 0 = default). */
cqg_status cqg_autotune_next(cqg_ctx *ctx);
/* Set which molecules of a batch take part in the following contractions (NULL: all);
 * a synchronous copy, to be called outside any captured region. */
cqg_status cqg_set_active(cqg_ctx *ctx, const unsigned char *active);
cqg_status cqg_get_launch_shapes(cqg_ctx *ctx, int *cta_per_sm, int *warps_per_cta);
/* The same plus, per list, the work-queue chunk (the quartets one warp claims at a time:
 * per-thread kernels in units of 32, one per lane; warp-cooperative kernels one after the
 * other) and the kernel form (1 = warp-cooperative, 0 = one quartet per thread; classes
 * that have both forms get theirs from the autotuner).  For the sibling-entry lists, warps
 * per CTA 2 selects CTAs of 64 threads (otherwise 128).  Any output may be NULL; 0 in the
 * first three = default. */
cqg_status cqg_get_schedule(cqg_ctx *ctx, int *cta_per_sm, int *warps_per_cta, int *quartets_per_warp,
                            int *warp_form);
/* Class fusion: tier 0 launches one kernel per class list; tier 1 evaluates the lists of
 * (ss|ss) and (ps|ss), tier 2 those of every
 * per-thread class up to (dd|dd), FP64 and FP32 alike, in one persistent kernel that pulls
 * chunks of every list from one device work queue; the other classes keep their own
 * launches.  The autotuner (cqg_autotune_next) times the three forms and keeps the fastest;
 * cqg_get_fusion returns the tier in use and the autotuner's times of tiers 0, 1, 2 (ms;
 * zero before tuning).  No reference counterpart (the reference's loop is one OpenMP
 * round-robin over all quartets, aointegrals_contract.h:107). */
cqg_status cqg_set_fusion(cqg_ctx *ctx, int tier);
cqg_status cqg_get_fusion(cqg_ctx *ctx, int *tier, double *tuned_ms);
/* Set the schedule of every list from arrays laid out as cqg_get_schedule's (NULL leaves
 * that part unchanged; the kernel form is taken only for classes that have both forms):
 * a schedule tuned once can be given to other contexts of the same system.  Entries out of
 * range (CTAs per SM above 64, warps per CTA above 4, quartets per warp above 1024, a form
 * other than 0 or 1) give CQG_ERR_BAD_ARG and change nothing. */
cqg_status cqg_set_schedule(cqg_ctx *ctx, const int *cta_per_sm, const int *warps_per_cta,
                            const int *quartets_per_warp, const int *warp_form);

/* Sibling groups (off by default).  Shell pairs whose shells share centres, angular momenta
 * and primitive exponents -- the segmented shells of one general contraction, such as the
 * 1s and 2s shells of cc-pVXZ oxygen -- differ only in their contraction coefficients.  With
 * siblings on, the classes (ss|ss), (ps|ss), (ps|ps), (pp|ss) and (ds|ss) get a second pair
 * of work lists of sibling entries: a bra and a ket group of such pairs with a mask of the
 * member quartets that pass the screen, evaluated from one pass over the groups' shared
 * primitive pairs.  The quartets evaluated, their count, their precision and their digest are
 * those of the pair-level lists; only the primitive work is shared.  The reference
 * evaluates every shell quartet from its own primitives (aointegrals_contract.h:133-140).
 * The schedule is kept (cqg_autotune_next retunes it for the changed lists); a CUDA graph
 * captured before the change must be captured again. */
cqg_status cqg_set_siblings(cqg_ctx *ctx, int on);
cqg_status cqg_get_siblings(cqg_ctx *ctx, int *on);
/* Sibling class k: a pair of sibling groups becomes one sibling entry when it holds at least
 * min_members member quartets (2..16; default half of the class's sibling form, 8 for
 * (ss|ss)); the member quartets of smaller pairs of groups are pair entries. */
cqg_status cqg_set_sibling_min(cqg_ctx *ctx, int k, int min_members);

/* Statistics of the last contraction (synchronises the context's stream). */
cqg_status cqg_get_stats(cqg_ctx *ctx, cqg_stats *out);
/* Largest number of entries held in the device quartet list at once (10 bytes each;
 * default 2^32, 40 GiB; an entry is one quartet, or one sibling-group quartet).  Larger
 * screened sets are filled and evaluated in chunks. */
cqg_status cqg_set_list_budget(cqg_ctx *ctx, long long quartets);
/* Per-class kernel timing on (1) / off (0, default). */
cqg_status cqg_set_timing(cqg_ctx *ctx, int on);
/* Name of quartet class index k ("(pp|ps)"), or NULL past the last class. */
const char *cqg_class_name(int k);
/* Work lists of the schedule arrays (cqg_get_schedule / cqg_set_schedule /
 * cqg_get_launch_shapes): 4 x 55 = 220, list b = part * 55 + class, parts: the FP64 and the
 * FP32 pair entries of each class, then its FP64 and FP32 sibling entries (cqg_set_siblings;
 * empty for the classes without them).  cqg_list_class gives list b's quartet class (-1 out
 * of range). */
int cqg_schedule_lists(void);
int cqg_list_class(int b);

/* ---- Kernels of the learned initial-density model (csrc/mlp.cu) ----
 * BF16 operands, FP32 accumulation; all pointers are device pointers, work is enqueued on
 * `stream`.  cqg_mlp_gemm_bf16: C(m,n) (+)= sum_k A[m*sam + k*sak] * B[n*sbn + k*sbk]
 * (accumulate != 0 adds into C), then if bias: C += bias[n]; if Y: Y = act ? SiLU(C) : C
 * in BF16 (leading dimension ldy).  cqg_mlp_silu_bwd: dZ = dY * SiLU'(Z) (BF16).
 * cqg_mlp_colsum: db[n] = sum_m dZ[m][n].  cqg_mlp_mse: *loss += sum mask (p-t)^2 * inv_count,
 * dpred = 2 mask (p-t) inv_count.  cqg_mlp_adam: one Adam step (bias-corrected, decoupled
 * weight decay folded into the gradient) on FP32 weights, optional BF16 copy.
 * These have no counterpart in the reference (it has no learned guess). */
cqg_status cqg_mlp_gemm_bf16(const void *A, long long sam, long long sak, const void *B,
                             long long sbn, long long sbk, float *C, long long ldc, int M, int N,
                             int K, const float *bias, void *Y, long long ldy, int act,
                             int accumulate, void *stream);
cqg_status cqg_mlp_silu_bwd(const float *dY, const float *Z, void *dZ, long long n, void *stream);
cqg_status cqg_mlp_to_bf16(const float *x, void *y, long long n, void *stream);
cqg_status cqg_mlp_colsum(const void *dZ, int M, int N, float *db, void *stream);
cqg_status cqg_mlp_mse(const float *pred, const float *target, const float *mask, long long n,
                       float inv_count, float *dpred, float *loss, void *stream);
cqg_status cqg_mlp_adam(float *w, const float *g, float *m1, float *m2, long long n, float lr,
                        float b1, float b2, float eps, int step, float weight_decay, void *wbf,
                        void *stream);
/* cqg_mlp_adam with the learning rate and the bias corrections read on the device from
 * hyper = {lr, 1 - b1^step, 1 - b2^step} (device pointer): the call can be captured in a
 * CUDA graph and replayed with a per-step schedule. */
cqg_status cqg_mlp_adam_dev(float *w, const float *g, float *m1, float *m2, long long n,
                            const float *hyper, float b1, float b2, float eps, float weight_decay,
                            void *wbf, void *stream);

/* FP64 / FP32 FMA throughput probe used to report roofline fractions: runs a dependent
 * FMA chain kernel for `ms_target` ms and returns achieved TFLOP/s in *tflops. */
cqg_status cqg_probe_fma_peak(int device, int fp64, double ms_target, double *tflops);

#ifdef __cplusplus
}
#endif
#endif /* CQGPU_H */
