// cqgpu engine: direct-SCF two-electron contraction G[X] = J - K on sm_100a.
//
// Data flow of one contraction (the reference loop it replaces is
// include/aointegrals/aointegrals_contract.h:24-194):
//   1. k_blocknorm   : M(s1,s2) = max_i max|X_i block|  (computeShBlkNorm, basisset.h:495-509),
//                      plus non-finite / asymmetry flags.
//   2. k_quartet_count / scan / k_quartet_fill : the unique shell quartets that pass the
//                      density-weighted Schwarz screen (contract.h:112-131), grouped by
//                      angular-momentum class, bra-major, as (bra pair, ket pair) indices.
//   3. k_eri_jk<class> : one thread per quartet: McMurchie-Davidson ERIs (generated code)
//                      and the J/K digest of contract.h:145-171 (half of the updates; the
//                      other half is the transpose) with FP64 atomics into Gh.
//   4. k_finalize    : AX += 0.5 (Gh + Gh^T)   (the 0.5*scale reduction of contract.h:189-193;
//                      the scales are folded into the digest).
#include "engine_impl.cuh"
#include "one_e.cuh"
#include "siblings.h"

static const char *kLetters = "spdfg";
static char g_class_names[55][16];
static bool g_names_init = false;

// MD-v1 model FLOPs per primitive quartet and per quartet digest, for class (la lb|lc ld).
static double md_v1_prim_flops(int la, int lb, int lc, int ld) {
  int p = la + lb, q = lc + ld, L = p + q;
  double c4 = (double)(L + 4) * (L + 3) * (L + 2) * (L + 1) / 24.0;
  return 30.0 + 3.0 * L + 2.0 * c4 + 2.0 * ncart_c(lc) * ncart_c(ld) * nherm_c(p) * nherm_c(q) +
         2.0 * ncart_c(la) * ncart_c(lb) * ncart_c(lc) * ncart_c(ld) * nherm_c(p);
}
static double md_v1_digest_flops(int la, int lb, int lc, int ld) {
  return 24.0 * nfun(la) * nfun(lb) * nfun(lc) * nfun(ld);
}

static double host_boys_row(int nmax, long double T, double *F) {
  long double term = 1.0L / (2 * nmax + 1), sum = term;
  for (int k = 1; k < 2000; k++) {
    term *= 2.0L * T / (2 * nmax + 2 * k + 1);
    sum += term;
    if (term < sum * 1e-22L) break;
  }
  long double ex = expl(-T);
  long double f = ex * sum;
  F[nmax] = (double)f;
  for (int m = nmax - 1; m >= 0; m--) {
    f = (2.0L * T * f + ex) / (2 * m + 1);
    F[m] = (double)f;
  }
  return 0;
}

// Primitive pairs of shell pair (a, b); prim_thresh = 0 keeps all of them, otherwise a
// pair whose s-type bound sqrt((ij|ij)) (with a (1+|AB|)^(la+lb) allowance) is below
// prim_thresh is dropped.
static void pair_prims(const cqg_ctx *ctx, int a, int b, double prim_thresh, std::vector<PrimPair> &out) {
  const double pi = 3.14159265358979323846;
  const double s2pi52 = std::sqrt(2.0 * std::pow(pi, 2.5));
  const double *A = &ctx->hcent[3 * a], *B = &ctx->hcent[3 * b];
  double AB2 = 0;
  for (int x = 0; x < 3; ++x) AB2 += (A[x] - B[x]) * (A[x] - B[x]);
  const double ABn = std::sqrt(AB2);
  for (int ia = 0; ia < ctx->hnprim[a]; ++ia)
    for (int ib = 0; ib < ctx->hnprim[b]; ++ib) {
      double al = ctx->halpha[ctx->hpoff[a] + ia], be = ctx->halpha[ctx->hpoff[b] + ib];
      double ca = ctx->hcoef[ctx->hpoff[a] + ia], cb = ctx->hcoef[ctx->hpoff[b] + ib];
      double p = al + be;
      double K = ca * cb * std::exp(-al * be / p * AB2);
      if (prim_thresh > 0) {
        double bound = std::fabs(K) * s2pi52 / (p * std::pow(2.0 * p, 0.25)) * std::pow(1.0 + ABn, ctx->hL[a] + ctx->hL[b]);
        if (bound < prim_thresh) continue;
      }
      PrimPair pp;
      pp.p = p;
      pp.ip = 1.0 / p;
      pp.Kp = s2pi52 * K / p;
      pp.Px = (al * A[0] + be * B[0]) / p;
      pp.Py = (al * A[1] + be * B[1]) / p;
      pp.Pz = (al * A[2] + be * B[2]) / p;
      out.push_back(pp);
    }
}

// primitive-count bucket of a shell pair: warps of the ERI kernels see kets of one bucket
static inline int prim_bucket(int np) {
  static const int upper[CQG_NBUCKET - 1] = {1, 2, 3, 4, 6, 8, 10, 12, 16, 20, 24, 32, 40, 48, 64};
  for (int b = 0; b < CQG_NBUCKET - 1; ++b)
    if (np <= upper[b]) return b;
  return CQG_NBUCKET - 1;
}

// build primitive-pair data for the current pair ordering and upload all pair arrays
static cqg_status upload_pairs(cqg_ctx *ctx, double prim_thresh) {
  size_t np = ctx->pair_sh.size();
  std::vector<int> poff(np), npr(np), kk(np);
  std::vector<PrimPair> prim;
  prim.reserve(np * 4);
  for (size_t i = 0; i < np; ++i) {
    int a = ctx->pair_sh[i].x, b = ctx->pair_sh[i].y;
    poff[i] = (int)prim.size();
    kk[i] = ctx->hnprim[a] * ctx->hnprim[b];
    pair_prims(ctx, a, b, prim_thresh, prim);
    npr[i] = (int)prim.size() - poff[i];
  }
  ctx->prim_pairs_total = (long long)prim.size();
  ctx->pair_np_host = npr;
  if (ctx->d_pair_sh.reserve(np) || ctx->d_pair_Q.reserve(np) || ctx->d_pair_poff.reserve(np) ||
      ctx->d_pair_np.reserve(np) || ctx->d_pair_kk.reserve(np) || ctx->d_prim.reserve(prim.size())) {
    ctx->err = "device allocation for pair data failed";
    return CQG_ERR_OOM;
  }
  CUCHK(cudaMemcpy(ctx->d_pair_sh.p, ctx->pair_sh.data(), np * sizeof(int2), cudaMemcpyHostToDevice));
  CUCHK(cudaMemcpy(ctx->d_pair_Q.p, ctx->pair_Q.data(), np * sizeof(double), cudaMemcpyHostToDevice));
  CUCHK(cudaMemcpy(ctx->d_pair_poff.p, poff.data(), np * sizeof(int), cudaMemcpyHostToDevice));
  CUCHK(cudaMemcpy(ctx->d_pair_np.p, npr.data(), np * sizeof(int), cudaMemcpyHostToDevice));
  CUCHK(cudaMemcpy(ctx->d_pair_kk.p, kk.data(), np * sizeof(int), cudaMemcpyHostToDevice));
  if (!prim.empty())
    CUCHK(cudaMemcpy(ctx->d_prim.p, prim.data(), prim.size() * sizeof(PrimPair), cudaMemcpyHostToDevice));
  return CQG_OK;
}

// Unit-coefficient primitive pairs of a sibling group and its members' coefficient
// products.  members[0] leads the group; the primitive pair (ia, ib) couples primitive ia of
// the leader's first shell with primitive ib of its second (the members share the
// exponents).  A primitive pair is kept when any member's bound |c_a c_b K| of pair_prims
// reaches prim_thresh (the union of the members' screened primitive pairs).  w gets `rows`
// rows, one value per kept primitive pair: row k = member k's products c_a(ia) c_b(ib), zero
// for the rows past the last member.
static void group_prims(const cqg_ctx *ctx, const int *members, int m, int rows, double prim_thresh,
                        const std::vector<int> &fam, std::vector<PrimPair> &out, std::vector<double> &w) {
  const double pi = 3.14159265358979323846;
  const double s2pi52 = std::sqrt(2.0 * std::pow(pi, 2.5));
  const int a = ctx->pair_sh[members[0]].x, b = ctx->pair_sh[members[0]].y;
  const double *A = &ctx->hcent[3 * a], *B = &ctx->hcent[3 * b];
  double AB2 = 0;
  for (int x = 0; x < 3; ++x) AB2 += (A[x] - B[x]) * (A[x] - B[x]);
  const double ABn = std::sqrt(AB2);
  // coefficient arrays of each member, in the leader's shell order
  std::vector<const double *> ca(m), cb(m);
  for (int k = 0; k < m; ++k) {
    const int x = ctx->pair_sh[members[k]].x, y = ctx->pair_sh[members[k]].y;
    const bool same = cqg_sib::same_orientation(x, a, fam);
    ca[k] = &ctx->hcoef[ctx->hpoff[same ? x : y]];
    cb[k] = &ctx->hcoef[ctx->hpoff[same ? y : x]];
  }
  std::vector<std::vector<double>> wk(rows);
  for (int ia = 0; ia < ctx->hnprim[a]; ++ia)
    for (int ib = 0; ib < ctx->hnprim[b]; ++ib) {
      const double al = ctx->halpha[ctx->hpoff[a] + ia], be = ctx->halpha[ctx->hpoff[b] + ib];
      const double p = al + be;
      const double K = std::exp(-al * be / p * AB2);
      bool keep = prim_thresh <= 0;
      if (!keep) {
        const double f = s2pi52 / (p * std::pow(2.0 * p, 0.25)) * std::pow(1.0 + ABn, ctx->hL[a] + ctx->hL[b]);
        for (int k = 0; k < m && !keep; ++k) keep = std::fabs(ca[k][ia] * cb[k][ib] * K) * f >= prim_thresh;
      }
      if (!keep) continue;
      PrimPair pp;
      pp.p = p;
      pp.ip = 1.0 / p;
      pp.Kp = s2pi52 * K / p;
      pp.Px = (al * A[0] + be * B[0]) / p;
      pp.Py = (al * A[1] + be * B[1]) / p;
      pp.Pz = (al * A[2] + be * B[2]) / p;
      out.push_back(pp);
      for (int k = 0; k < rows; ++k) wk[k].push_back(k < m ? ca[k][ia] * cb[k][ib] : 0.0);
    }
  for (int k = 0; k < rows; ++k) w.insert(w.end(), wk[k].begin(), wk[k].end());
}

// Quartet class k has the sibling form (its lists hold group entries when siblings are on).
static bool class_grouped(int k) {
  static bool table[CQG_NQC];
  static bool init = false;
  if (!init) {
    for (int q = 0; q < CQG_NQC; ++q) table[q] = false;
#define CQG_GC_MARK(A, B, C, D, MB, MK) \
  table[pair_class_of(A, B) * (pair_class_of(A, B) + 1) / 2 + pair_class_of(C, D)] = true;
    CQG_GC_EACH(CQG_GC_MARK)
#undef CQG_GC_MARK
    init = true;
  }
  return k >= 0 && k < CQG_NQC && table[k];
}

// Default smallest member count of a sibling entry: half of the sibling form's MB x MK
// quartets (a pair of groups that fills less of the form runs as separate pair quartets).
static int default_sibling_min(int k) {
#define CQG_GC_MIN(A, B, C, D, MB, MK) \
  if (k == pair_class_of(A, B) * (pair_class_of(A, B) + 1) / 2 + pair_class_of(C, D)) return (MB * MK + 1) / 2;
  CQG_GC_EACH(CQG_GC_MIN)
#undef CQG_GC_MIN
  return 0;
}

// Pair classes that are the bra or ket of a sibling class (their pairs get group data).
static bool pair_class_in_groups(int c) {
  for (int k = 0; k < CQG_NQC; ++k) {
    if (!class_grouped(k)) continue;
    int i, j;
    qclass_split(k, i, j);
    if (i == c || j == c) return true;
  }
  return false;
}

// Group data of the current pair order (leaders: unit primitive pairs and member weights)
// and the group index arrays, to the device.
static cqg_status upload_groups(cqg_ctx *ctx, const std::vector<int> &fam, double prim_thresh) {
  const int np = (int)ctx->pair_sh.size();
  std::vector<int> gpoff(np, 0), gnp(np, 0), gwoff(np, 0);
  std::vector<PrimPair> prim;
  std::vector<double> w;
  std::vector<int> members;
  for (int c = 0; c < CQG_NPC; ++c) {
    if (!pair_class_in_groups(c)) continue;
    const int rows = sibling_cap(kPairClass[c][0], kPairClass[c][1]);
    for (int i = ctx->pc_beg[c]; i < ctx->pc_beg[c + 1]; ++i) {
      const int m = ctx->pair_gsz[i];
      if (m == 0) continue;   // not a leader
      members.resize(m);
      for (int k = 0; k < m; ++k) members[k] = i + k;
      gpoff[i] = (int)prim.size();
      gwoff[i] = (int)w.size();
      group_prims(ctx, members.data(), m, rows, prim_thresh, fam, prim, w);
      gnp[i] = (int)prim.size() - gpoff[i];
    }
  }
  const size_t ng = ctx->glead.size();
  if (ctx->d_pair_Qc.reserve(np) || ctx->d_gsz.reserve(np) || ctx->d_gpoff.reserve(np) || ctx->d_gnp.reserve(np) ||
      ctx->d_gwoff.reserve(np) || ctx->d_gprim.reserve(std::max<size_t>(prim.size(), 1)) ||
      ctx->d_gw.reserve(std::max<size_t>(w.size(), 1)) || ctx->d_glead.reserve(std::max<size_t>(ng, 1)) ||
      ctx->d_gQ.reserve(std::max<size_t>(ng, 1))) {
    ctx->err = "device allocation for sibling-group data failed";
    return CQG_ERR_OOM;
  }
  CUCHK(cudaMemcpy(ctx->d_pair_Qc.p, ctx->pair_Qc.data(), np * sizeof(double), cudaMemcpyHostToDevice));
  CUCHK(cudaMemcpy(ctx->d_gsz.p, ctx->pair_gsz.data(), np * sizeof(int), cudaMemcpyHostToDevice));
  CUCHK(cudaMemcpy(ctx->d_gpoff.p, gpoff.data(), np * sizeof(int), cudaMemcpyHostToDevice));
  CUCHK(cudaMemcpy(ctx->d_gnp.p, gnp.data(), np * sizeof(int), cudaMemcpyHostToDevice));
  CUCHK(cudaMemcpy(ctx->d_gwoff.p, gwoff.data(), np * sizeof(int), cudaMemcpyHostToDevice));
  if (!prim.empty())
    CUCHK(cudaMemcpy(ctx->d_gprim.p, prim.data(), prim.size() * sizeof(PrimPair), cudaMemcpyHostToDevice));
  if (!w.empty()) CUCHK(cudaMemcpy(ctx->d_gw.p, w.data(), w.size() * sizeof(double), cudaMemcpyHostToDevice));
  if (ng) {
    CUCHK(cudaMemcpy(ctx->d_glead.p, ctx->glead.data(), ng * sizeof(int), cudaMemcpyHostToDevice));
    CUCHK(cudaMemcpy(ctx->d_gQ.p, ctx->gQ.data(), ng * sizeof(double), cudaMemcpyHostToDevice));
  }
  ctx->group_prim_pairs = (long long)prim.size();
  return CQG_OK;
}

// The active block table: bra-group tasks for the sibling classes, or pair tasks for all.
static void select_block_table(cqg_ctx *ctx) {
  ctx->bt = ctx->siblings ? ctx->bt_group : ctx->bt_pair;
  ctx->ntask = ctx->siblings ? ctx->ntask_group : ctx->ntask_pair;
}

// Class-block tables: pair tasks for every class (bt_pair), and bra-group tasks for the
// sibling classes (bt_group); then the active one.  The per-task count and offset arrays
// are sized for the larger of the two.
static cqg_status build_block_tables(cqg_ctx *ctx) {
  for (int mode = 0; mode < 2; ++mode) {
    BlockTable &bt = mode ? ctx->bt_group : ctx->bt_pair;
    memset(&bt, 0, sizeof(bt));
    int task = 0;
    for (int k = 0; k < CQG_NQC; ++k) {
      int i, j;
      qclass_split(k, i, j);
      bt.task_beg[k] = task;
      bt.bra_beg[k] = ctx->pc_beg[i];
      bt.ket_beg[k] = ctx->pc_beg[j];
      bt.ket_n[k] = ctx->pc_beg[j + 1] - ctx->pc_beg[j];
      bt.ket_class[k] = j;
      bt.diag[k] = (i == j);
      bt.grouped[k] = mode == 1 && class_grouped(k) && ctx->sibling_min[k] > 0;
      bt.gbra_beg[k] = ctx->gc_beg[i];
      bt.min_members[k] = ctx->sibling_min[k];
      task += bt.grouped[k] ? ctx->gc_beg[i + 1] - ctx->gc_beg[i] : ctx->pc_beg[i + 1] - ctx->pc_beg[i];
    }
    bt.task_beg[CQG_NQC] = task;
    bt.nblk = CQG_NQC;
    (mode ? ctx->ntask_group : ctx->ntask_pair) = task;
  }
  select_block_table(ctx);
  const size_t task = (size_t)std::max(ctx->ntask_pair, ctx->ntask_group);
  size_t scan_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (long long *)nullptr, (long long *)nullptr,
                                std::max<int>(kListParts * (int)task, 1));
  if (ctx->d_cnt.reserve(kListParts * task + 1) || ctx->d_off.reserve(kListParts * task + 1) ||
      ctx->d_scan_tmp.reserve(scan_bytes + 16) || ctx->d_mslot.reserve(task + 1) || ctx->d_mhead.reserve(1) ||
      ctx->d_masks.reserve(kMaskStepsInitial))
    return CQG_ERR_OOM;
  return CQG_OK;
}


// Launchers of every quartet class (eri_part.cu, a share per translation unit), merged
// into one table per precision.
#define CQG_SHARE_DECL(k)                                 \
  const eri_launcher *cqg_eri_part_table_##k(int fp32); \
  const eri_launcher *cqg_eri_part_gc_table_##k(int fp32);
CQG_SHARE_DECL(0)
CQG_SHARE_DECL(1)
CQG_SHARE_DECL(2)
CQG_SHARE_DECL(3)
CQG_SHARE_DECL(4)
CQG_SHARE_DECL(5)
CQG_SHARE_DECL(6)
CQG_SHARE_DECL(7)
#undef CQG_SHARE_DECL
static_assert(CQG_NPART == 8, "one table accessor per share");
static const eri_launcher *cqg_eri_part_table(int part, int fp32) {
  switch (part) {
    case 0: return cqg_eri_part_table_0(fp32);
    case 1: return cqg_eri_part_table_1(fp32);
    case 2: return cqg_eri_part_table_2(fp32);
    case 3: return cqg_eri_part_table_3(fp32);
    case 4: return cqg_eri_part_table_4(fp32);
    case 5: return cqg_eri_part_table_5(fp32);
    case 6: return cqg_eri_part_table_6(fp32);
    default: return cqg_eri_part_table_7(fp32);
  }
}
static const eri_launcher *cqg_eri_part_gc_table(int part, int fp32) {
  switch (part) {
    case 0: return cqg_eri_part_gc_table_0(fp32);
    case 1: return cqg_eri_part_gc_table_1(fp32);
    case 2: return cqg_eri_part_gc_table_2(fp32);
    case 3: return cqg_eri_part_gc_table_3(fp32);
    case 4: return cqg_eri_part_gc_table_4(fp32);
    case 5: return cqg_eri_part_gc_table_5(fp32);
    case 6: return cqg_eri_part_gc_table_6(fp32);
    default: return cqg_eri_part_gc_table_7(fp32);
  }
}
// launcher of every work list vb = part * CQG_NQC + class: the class kernels (FP64, FP32)
// for the pair entries, the sibling-group kernels (FP64, FP32; null for the other classes)
// for the sibling entries
struct EriTables {
  eri_launcher t[CQG_NLIST];
  EriTables() {
    for (int k = 0; k < CQG_NQC; ++k) {
      t[k] = cqg_eri_part_table(k % CQG_NPART, 0)[k];
      t[CQG_NQC + k] = cqg_eri_part_table(k % CQG_NPART, 1)[k];
      t[2 * CQG_NQC + k] = cqg_eri_part_gc_table(k % CQG_NPART, 0)[k];
      t[3 * CQG_NQC + k] = cqg_eri_part_gc_table(k % CQG_NPART, 1)[k];
    }
  }
};
static const EriTables kEriTables;
static const eri_launcher *const kEriLaunch = kEriTables.t;      // FP64 class lists
static const eri_launcher *const kEriLaunch32 = kEriTables.t + CQG_NQC;
static inline eri_launcher list_launcher(int vb) { return kEriTables.t[vb]; }

extern "C" {

const char *cqg_version(void) { return "cqgpu 0.1 (sm_100a, MD FP64)"; }

const char *cqg_status_string(cqg_status s) {
  switch (s) {
    case CQG_OK: return "ok";
    case CQG_ERR_BAD_ARG: return "bad argument";
    case CQG_ERR_OOM: return "out of device memory";
    case CQG_ERR_CUDA: return "CUDA error";
    case CQG_ERR_TIMEOUT: return "device wait timed out";
    case CQG_ERR_NONFINITE: return "non-finite input";
    case CQG_ERR_STATE: return "invalid call order";
    case CQG_ERR_UNSUPPORTED: return "unsupported input";
  }
  return "unknown status";
}

int cqg_schedule_lists(void) { return CQG_NLIST; }

int cqg_list_class(int b) {
  if (b < 0 || b >= CQG_NLIST) return -1;
  return b % CQG_NQC;
}

const char *cqg_class_name(int k) {
  if (!g_names_init) {
    for (int q = 0; q < 55; ++q) {
      int i, j;
      qclass_split(q, i, j);
      snprintf(g_class_names[q], 16, "(%c%c|%c%c)", kLetters[kPairClass[i][0]], kLetters[kPairClass[i][1]],
               kLetters[kPairClass[j][0]], kLetters[kPairClass[j][1]]);
    }
    g_names_init = true;
  }
  if (k < 0 || k >= CQG_NQC) return nullptr;
  return g_class_names[k];
}

cqg_status cqg_create(cqg_ctx **out, int device) {
  if (!out) return CQG_ERR_BAD_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return CQG_ERR_CUDA;
  cqg_ctx *ctx = new cqg_ctx();
  ctx->device = device;
  memset(&ctx->stats, 0, sizeof(ctx->stats));
  if (cudaSetDevice(device) != cudaSuccess) {
    delete ctx;
    return CQG_ERR_CUDA;
  }
  // Boys table
  std::vector<double> tab(BOYS_TABLE_SIZE);
  for (int i = 0; i < BOYS_NT; ++i) host_boys_row(BOYS_NORD - 1, (long double)i / 10.0L, &tab[i * BOYS_NORD]);
  for (int i = 0; i < BOYS_NT; ++i) tab[BOYS_NT * BOYS_NORD + i] = (double)expl(-(long double)i / 10.0L);
  if (ctx->d_boys.reserve(tab.size()) != cudaSuccess ||
      cudaMemcpy(ctx->d_boys.p, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
    delete ctx;
    return CQG_ERR_CUDA;
  }
  for (int i = 0; i < 4 + 2 * CQG_NQC + 2; ++i) cudaEventCreate(&ctx->ev[i]);
  for (int k = 0; k < CQG_NQC; ++k) ctx->sibling_min[k] = default_sibling_min(k);
  ctx->events = true;
  cudaDeviceGetAttribute(&ctx->nsm, cudaDevAttrMultiProcessorCount, device);
  *out = ctx;
  return CQG_OK;
}

cqg_status cqg_destroy(cqg_ctx *ctx) {
  if (!ctx) return CQG_OK;
  cudaSetDevice(ctx->device);
  ctx->d_center.release(); ctx->d_bf.release(); ctx->d_sz.release();
  ctx->d_pair_sh.release(); ctx->d_pair_Q.release(); ctx->d_pair_poff.release(); ctx->d_pair_np.release();
  ctx->d_pair_kk.release(); ctx->d_blkacc.release();
  ctx->d_shL.release(); ctx->d_shnp.release(); ctx->d_shpoff.release(); ctx->d_alpha.release();
  ctx->d_coef.release(); ctx->d_allpairs.release(); ctx->d_oe.release(); ctx->d_charges.release();
  ctx->d_shmol.release(); ctx->d_mshoff.release(); ctx->d_mnsh.release(); ctx->d_mnbf.release();
  ctx->d_molbk.release(); ctx->d_mxoff.release(); ctx->d_mMoff.release(); ctx->d_active.release();
  ctx->d_prim.release(); ctx->d_boys.release();
  ctx->d_M.release(); ctx->d_Mmax.release(); ctx->d_Mpair.release(); ctx->d_flags.release();
  ctx->d_cnt.release(); ctx->d_off.release(); ctx->d_range.release(); ctx->d_scan_tmp.release();
  ctx->d_qhead.release();
  ctx->d_qlist.release(); ctx->d_G.release(); ctx->d_X.release(); ctx->d_AX.release(); ctx->d_Gscratch.release();
  ctx->d_molgbk.release(); ctx->d_gsz.release(); ctx->d_gpoff.release(); ctx->d_gnp.release(); ctx->d_gwoff.release();
  ctx->d_glead.release(); ctx->d_pair_Qc.release(); ctx->d_gQ.release(); ctx->d_gw.release(); ctx->d_gprim.release();
  ctx->d_qmask.release(); ctx->d_masks.release(); ctx->d_mhead.release(); ctx->d_mslot.release();
  if (ctx->events)
    for (int i = 0; i < 4 + 2 * CQG_NQC + 2; ++i) cudaEventDestroy(ctx->ev[i]);
  delete ctx;
  return CQG_OK;
}

const char *cqg_last_error(const cqg_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

cqg_status cqg_set_threshold(cqg_ctx *ctx, double thresh) {
  if (!ctx || !(thresh >= 0.0)) return CQG_ERR_BAD_ARG;
  ctx->thresh = thresh;
  return CQG_OK;
}

cqg_status cqg_set_precision(cqg_ctx *ctx, int policy, double cutoff) {
  if (!ctx || (policy != CQG_PREC_FP64 && policy != CQG_PREC_MIXED) || !(cutoff >= 0.0)) return CQG_ERR_BAD_ARG;
  ctx->policy = policy;
  ctx->fp32_cutoff = cutoff;
  return CQG_OK;
}

cqg_status cqg_set_list_budget(cqg_ctx *ctx, long long quartets) {
  if (!ctx || quartets < 1) return CQG_ERR_BAD_ARG;
  ctx->list_budget = quartets;
  return CQG_OK;
}

cqg_status cqg_set_timing(cqg_ctx *ctx, int on) {
  if (!ctx) return CQG_ERR_BAD_ARG;
  ctx->timing = on ? 1 : 0;
  return CQG_OK;
}

cqg_status cqg_get_sizes(cqg_ctx *ctx, int *nshell, int *nbasis, int *maxl) {
  if (!ctx) return CQG_ERR_BAD_ARG;
  if (nshell) *nshell = ctx->nshell;
  if (nbasis) *nbasis = ctx->nbf;
  if (maxl) *maxl = ctx->maxl;
  return CQG_OK;
}

cqg_status cqg_set_basis_batch(cqg_ctx *ctx, int nmol, const int *nshell_per_mol, const int *L, const int *pure,
                               const int *nprim, const double *alpha, const double *coef, const double *centers) {
  if (!ctx || nmol <= 0 || !nshell_per_mol || !L || !pure || !nprim || !alpha || !coef || !centers)
    return CQG_ERR_BAD_ARG;
  CUCHK(cudaSetDevice(ctx->device));
  int nshell = 0;
  for (int m = 0; m < nmol; ++m) {
    if (nshell_per_mol[m] <= 0) {
      ctx->err = "molecule without shells";
      return CQG_ERR_BAD_ARG;
    }
    nshell += nshell_per_mol[m];
  }
  int tot = 0, maxl = 0;
  for (int s = 0; s < nshell; ++s) {
    if (L[s] < 0 || nprim[s] <= 0) {
      ctx->err = "shell with negative L or no primitives";
      return CQG_ERR_BAD_ARG;
    }
    if (L[s] > CQG_MAXL) {
      ctx->err = "angular momentum above " + std::to_string(CQG_MAXL) + " is not built into this engine";
      return CQG_ERR_UNSUPPORTED;
    }
    if ((pure[s] != 0) != (L[s] > 1)) {
      ctx->err = "engine requires spherical shells exactly for L > 1 (the reference default)";
      return CQG_ERR_UNSUPPORTED;
    }
    tot += nprim[s];
    maxl = std::max(maxl, L[s]);
  }
  ctx->nmol = nmol;
  ctx->nshell = nshell;
  ctx->maxl = maxl;
  ctx->hL.assign(L, L + nshell);
  ctx->hnprim.assign(nprim, nprim + nshell);
  ctx->halpha.assign(alpha, alpha + tot);
  ctx->hcoef.assign(coef, coef + tot);
  ctx->hcent.assign(centers, centers + 3 * nshell);
  ctx->hbf.resize(nshell);
  ctx->hsz.resize(nshell);
  ctx->hpoff.resize(nshell);
  ctx->hshmol.resize(nshell);
  ctx->m_shoff.resize(nmol);
  ctx->m_nsh.resize(nmol);
  ctx->m_nbf.resize(nmol);
  ctx->m_xoff.resize(nmol);
  ctx->m_Moff.resize(nmol);
  {
    int p = 0, s = 0;
    long long xo = 0, mo = 0;
    ctx->max_nsh = 0;
    ctx->max_nbf = 0;
    for (int m = 0; m < nmol; ++m) {
      ctx->m_shoff[m] = s;
      ctx->m_nsh[m] = nshell_per_mol[m];
      int f = 0;
      for (int k = 0; k < nshell_per_mol[m]; ++k, ++s) {
        ctx->hbf[s] = f;
        ctx->hsz[s] = nfun(L[s]);
        f += ctx->hsz[s];
        ctx->hpoff[s] = p;
        p += nprim[s];
        ctx->hshmol[s] = m;
      }
      ctx->m_nbf[m] = f;
      ctx->m_xoff[m] = xo;
      ctx->m_Moff[m] = mo;
      xo += (long long)f * f;
      mo += (long long)nshell_per_mol[m] * nshell_per_mol[m];
      ctx->max_nsh = std::max(ctx->max_nsh, nshell_per_mol[m]);
      ctx->max_nbf = std::max(ctx->max_nbf, f);
    }
    ctx->packed = xo;
    ctx->Mtotal = mo;
  }
  ctx->nbf = ctx->m_nbf[0];
  // shells and molecule layout to device
  std::vector<double3> c3(nshell);
  for (int s = 0; s < nshell; ++s) c3[s] = make_double3(centers[3 * s], centers[3 * s + 1], centers[3 * s + 2]);
  if (ctx->d_center.reserve(nshell) || ctx->d_bf.reserve(nshell) || ctx->d_sz.reserve(nshell) ||
      ctx->d_shmol.reserve(nshell) || ctx->d_mshoff.reserve(nmol) || ctx->d_mnsh.reserve(nmol) ||
      ctx->d_mnbf.reserve(nmol) || ctx->d_mxoff.reserve(nmol) || ctx->d_mMoff.reserve(nmol) ||
      ctx->d_active.reserve(nmol))
    return CQG_ERR_OOM;
  CUCHK(cudaMemcpy(ctx->d_center.p, c3.data(), nshell * sizeof(double3), cudaMemcpyHostToDevice));
  CUCHK(cudaMemcpy(ctx->d_bf.p, ctx->hbf.data(), nshell * sizeof(int), cudaMemcpyHostToDevice));
  CUCHK(cudaMemcpy(ctx->d_sz.p, ctx->hsz.data(), nshell * sizeof(int), cudaMemcpyHostToDevice));
  CUCHK(cudaMemcpy(ctx->d_shmol.p, ctx->hshmol.data(), nshell * sizeof(int), cudaMemcpyHostToDevice));
  CUCHK(cudaMemcpy(ctx->d_mshoff.p, ctx->m_shoff.data(), nmol * sizeof(int), cudaMemcpyHostToDevice));
  CUCHK(cudaMemcpy(ctx->d_mnsh.p, ctx->m_nsh.data(), nmol * sizeof(int), cudaMemcpyHostToDevice));
  CUCHK(cudaMemcpy(ctx->d_mnbf.p, ctx->m_nbf.data(), nmol * sizeof(int), cudaMemcpyHostToDevice));
  CUCHK(cudaMemcpy(ctx->d_mxoff.p, ctx->m_xoff.data(), nmol * sizeof(long long), cudaMemcpyHostToDevice));
  CUCHK(cudaMemcpy(ctx->d_mMoff.p, ctx->m_Moff.data(), nmol * sizeof(long long), cudaMemcpyHostToDevice));
  ctx->h_active.assign(nmol, 1);
  CUCHK(cudaMemcpy(ctx->d_active.p, ctx->h_active.data(), nmol, cudaMemcpyHostToDevice));
  // raw shells (one-electron integrals) and the list of all pairs a >= b within each molecule
  {
    std::vector<int2> allp;
    for (int m = 0; m < nmol; ++m)
      for (int a = ctx->m_shoff[m]; a < ctx->m_shoff[m] + ctx->m_nsh[m]; ++a)
        for (int b = ctx->m_shoff[m]; b <= a; ++b) allp.push_back(make_int2(a, b));
    ctx->nallpairs = (long long)allp.size();
    if (ctx->d_shL.reserve(nshell) || ctx->d_shnp.reserve(nshell) || ctx->d_shpoff.reserve(nshell) ||
        ctx->d_alpha.reserve(tot) || ctx->d_coef.reserve(tot) || ctx->d_allpairs.reserve(allp.size()))
      return CQG_ERR_OOM;
    CUCHK(cudaMemcpy(ctx->d_shL.p, L, nshell * sizeof(int), cudaMemcpyHostToDevice));
    CUCHK(cudaMemcpy(ctx->d_shnp.p, nprim, nshell * sizeof(int), cudaMemcpyHostToDevice));
    CUCHK(cudaMemcpy(ctx->d_shpoff.p, ctx->hpoff.data(), nshell * sizeof(int), cudaMemcpyHostToDevice));
    CUCHK(cudaMemcpy(ctx->d_alpha.p, alpha, tot * sizeof(double), cudaMemcpyHostToDevice));
    CUCHK(cudaMemcpy(ctx->d_coef.p, coef, tot * sizeof(double), cudaMemcpyHostToDevice));
    CUCHK(cudaMemcpy(ctx->d_allpairs.p, allp.data(), allp.size() * sizeof(int2), cudaMemcpyHostToDevice));
  }
  // pairs within each molecule, by class, internal orientation L_a >= L_b (a >= b when equal L)
  std::vector<std::vector<int2>> bycls(CQG_NPC);
  for (int m = 0; m < nmol; ++m)
    for (int a = ctx->m_shoff[m]; a < ctx->m_shoff[m] + ctx->m_nsh[m]; ++a)
      for (int b = ctx->m_shoff[m]; b <= a; ++b) {
        int x = a, y = b;
        if (L[y] > L[x]) std::swap(x, y);
        bycls[pair_class_of(L[x], L[y])].push_back(make_int2(x, y));
      }
  ctx->pair_sh.clear();
  for (int c = 0; c < CQG_NPC; ++c) {
    ctx->pc_beg[c] = (int)ctx->pair_sh.size();
    ctx->pair_sh.insert(ctx->pair_sh.end(), bycls[c].begin(), bycls[c].end());
  }
  ctx->pc_beg[CQG_NPC] = (int)ctx->pair_sh.size();
  ctx->pair_Q.assign(ctx->pair_sh.size(), 0.0);
  cqg_status st = upload_pairs(ctx, 0.0);
  if (st != CQG_OK) return st;
  // Schwarz on the device with all primitive pairs (computeSchwartz uses precision 0)
  Pairs P = make_pairs(ctx);
  Shells S = make_shells(ctx);
  double *dQ = ctx->d_pair_Q.p;
  cudaError_t e = cudaSuccess;
  e = e ? e : launch_schwarz<0, 0>(ctx, P, S, ctx->pc_beg[0], ctx->pc_beg[1], dQ);
  e = e ? e : launch_schwarz<1, 0>(ctx, P, S, ctx->pc_beg[1], ctx->pc_beg[2], dQ);
  e = e ? e : launch_schwarz<1, 1>(ctx, P, S, ctx->pc_beg[2], ctx->pc_beg[3], dQ);
  e = e ? e : launch_schwarz<2, 0>(ctx, P, S, ctx->pc_beg[3], ctx->pc_beg[4], dQ);
  e = e ? e : launch_schwarz<2, 1>(ctx, P, S, ctx->pc_beg[4], ctx->pc_beg[5], dQ);
  e = e ? e : launch_schwarz<2, 2>(ctx, P, S, ctx->pc_beg[5], ctx->pc_beg[6], dQ);
  e = e ? e : launch_schwarz<3, 0>(ctx, P, S, ctx->pc_beg[6], ctx->pc_beg[7], dQ);
  e = e ? e : launch_schwarz<3, 1>(ctx, P, S, ctx->pc_beg[7], ctx->pc_beg[8], dQ);
  e = e ? e : launch_schwarz<3, 2>(ctx, P, S, ctx->pc_beg[8], ctx->pc_beg[9], dQ);
  e = e ? e : launch_schwarz<3, 3>(ctx, P, S, ctx->pc_beg[9], ctx->pc_beg[10], dQ);
  if (e != cudaSuccess) {
    ctx->err = std::string("schwarz kernels: ") + cudaGetErrorString(e);
    return CQG_ERR_CUDA;
  }
  CUCHK(cudaDeviceSynchronize());
  CUCHK(cudaMemcpy(ctx->pair_Q.data(), dQ, ctx->pair_Q.size() * sizeof(double), cudaMemcpyDeviceToHost));
  if (nmol == 1) {
    ctx->Qmat.assign((size_t)nshell * nshell, 0.0);
    for (size_t i = 0; i < ctx->pair_sh.size(); ++i) {
      int a = ctx->pair_sh[i].x, b = ctx->pair_sh[i].y;
      ctx->Qmat[a + (size_t)b * nshell] = ctx->pair_Q[i];
      ctx->Qmat[b + (size_t)a * nshell] = ctx->pair_Q[i];
    }
  } else {
    ctx->Qmat.clear();
  }
  // Sibling groups per pair class (csrc/siblings.h), their largest Q and the size of the
  // union of their members' screened primitive pairs.
  const int npairs = (int)ctx->pair_sh.size();
  const std::vector<int> fam = cqg_sib::shell_families(nshell, L, nprim, ctx->hpoff.data(), alpha, centers,
                                                       ctx->hshmol.data());
  std::vector<int> pgid(npairs), prank(npairs), gnp_of(npairs);   // gnp_of: by group id
  std::vector<double> gq_of(npairs, 0.0);
  {
    int gbase = 0;
    std::vector<int> pa, pb, gid, rank;
    for (int c = 0; c < CQG_NPC; ++c) {
      const int b0 = ctx->pc_beg[c], n = ctx->pc_beg[c + 1] - b0;
      pa.resize(n);
      pb.resize(n);
      for (int k = 0; k < n; ++k) {
        pa[k] = ctx->pair_sh[b0 + k].x;
        pb[k] = ctx->pair_sh[b0 + k].y;
      }
      const int cap = sibling_cap(kPairClass[c][0], kPairClass[c][1]);
      const int ng = cqg_sib::pair_groups(n, pa.data(), pb.data(), L, fam, cap, gid, rank);
      for (int k = 0; k < n; ++k) {
        pgid[b0 + k] = gbase + gid[k];
        prank[b0 + k] = rank[k];
      }
      gbase += ng;
    }
    std::vector<std::vector<int>> members(gbase);
    for (int i = 0; i < npairs; ++i) members[pgid[i]].push_back(i);
    std::vector<PrimPair> tmp;
    std::vector<double> w;
    for (int g = 0; g < gbase; ++g) {
      double q = 0.0;
      for (int i : members[g]) q = std::max(q, ctx->pair_Q[i]);
      gq_of[g] = q;
      tmp.clear();
      w.clear();
      group_prims(ctx, members[g].data(), (int)members[g].size(), 1, 1e-24, fam, tmp, w);
      gnp_of[g] = (int)tmp.size();
    }
  }
  // Sort each class by (molecule, primitive-count bucket of the group, group Q descending,
  // group, member), stable.  The members of a group become consecutive pairs led by the
  // first, and Qc (the group's Q) is non-increasing within each bucket.  Per (molecule,
  // class) bucket starts -> molbk (pair index) and molgbk (group index).
  auto bucket_of = [&](int i) { return prim_bucket(gnp_of[pgid[i]]); };
  const int NB1 = CQG_NBUCKET + 1;
  std::vector<int> molbk((size_t)nmol * CQG_NPC * NB1, 0), molgbk((size_t)nmol * CQG_NPC * NB1, 0);
  std::vector<int> new_gid(npairs);
  for (int c = 0; c < CQG_NPC; ++c) {
    int b0 = ctx->pc_beg[c], b1 = ctx->pc_beg[c + 1];
    std::vector<int> idx(b1 - b0);
    std::iota(idx.begin(), idx.end(), b0);
    std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) {
      int mx = ctx->hshmol[ctx->pair_sh[x].x], my = ctx->hshmol[ctx->pair_sh[y].x];
      if (mx != my) return mx < my;
      int bx = bucket_of(x), by = bucket_of(y);
      if (bx != by) return bx < by;
      const double qx = gq_of[pgid[x]], qy = gq_of[pgid[y]];
      if (qx != qy) return qx > qy;
      if (pgid[x] != pgid[y]) return pgid[x] < pgid[y];
      return prank[x] < prank[y];
    });
    // bucket starts per molecule: first index of (m, bk); empty buckets start where the next begins
    std::vector<int> first((size_t)nmol * NB1, -1);
    for (int k = 0; k < (int)idx.size(); ++k) {
      const int m = ctx->hshmol[ctx->pair_sh[idx[k]].x], bk = bucket_of(idx[k]);
      if (first[(size_t)m * NB1 + bk] < 0) first[(size_t)m * NB1 + bk] = b0 + k;
    }
    int next = b1;
    for (int m = nmol - 1; m >= 0; --m) {
      int *row = &molbk[((size_t)m * CQG_NPC + c) * NB1];
      row[CQG_NBUCKET] = next;
      for (int bk = CQG_NBUCKET - 1; bk >= 0; --bk) {
        const int f = first[(size_t)m * NB1 + bk];
        row[bk] = f >= 0 ? f : row[bk + 1];
      }
      next = row[0];
    }
    for (int bk = 0; bk <= CQG_NBUCKET; ++bk) ctx->bucket_beg[c][bk] = molbk[(size_t)c * NB1 + bk];
    std::vector<int2> sh2;
    std::vector<double> q2;
    std::vector<int> g2;
    for (int i : idx) {
      sh2.push_back(ctx->pair_sh[i]);
      q2.push_back(ctx->pair_Q[i]);
      g2.push_back(pgid[i]);
    }
    std::copy(sh2.begin(), sh2.end(), ctx->pair_sh.begin() + b0);
    std::copy(q2.begin(), q2.end(), ctx->pair_Q.begin() + b0);
    std::copy(g2.begin(), g2.end(), new_gid.begin() + b0);
  }
  // group index space in pair order: leaders, group sizes, Qc, bucket starts by group
  ctx->pair_gsz.assign(npairs, 0);
  ctx->pair_Qc.assign(npairs, 0.0);
  ctx->glead.clear();
  ctx->gQ.clear();
  {
    std::vector<int> pair_group(npairs);
    for (int i = 0; i < npairs; ++i) {
      if (i == 0 || new_gid[i] != new_gid[i - 1]) {
        ctx->glead.push_back(i);
        ctx->gQ.push_back(gq_of[new_gid[i]]);
      }
      pair_group[i] = (int)ctx->glead.size() - 1;
      ctx->pair_gsz[ctx->glead.back()] += 1;
      ctx->pair_Qc[i] = gq_of[new_gid[i]];
    }
    const int ngroups = (int)ctx->glead.size();
    for (int c = 0; c <= CQG_NPC; ++c) {
      const int pb = ctx->pc_beg[c];
      ctx->gc_beg[c] = pb < npairs ? pair_group[pb] : ngroups;
    }
    for (size_t k = 0; k < molbk.size(); ++k) molgbk[k] = molbk[k] < npairs ? pair_group[molbk[k]] : ngroups;
  }
  if (ctx->d_molbk.reserve(molbk.size()) || ctx->d_molgbk.reserve(molgbk.size())) return CQG_ERR_OOM;
  CUCHK(cudaMemcpy(ctx->d_molbk.p, molbk.data(), molbk.size() * sizeof(int), cudaMemcpyHostToDevice));
  CUCHK(cudaMemcpy(ctx->d_molgbk.p, molgbk.data(), molgbk.size() * sizeof(int), cudaMemcpyHostToDevice));
  st = upload_pairs(ctx, 1e-24);
  if (st != CQG_OK) return st;
  st = upload_groups(ctx, fam, 1e-24);
  if (st != CQG_OK) return st;
  {
    cqg_status bst = build_block_tables(ctx);
    if (bst != CQG_OK) return bst;
  }
  const int task = std::max(ctx->ntask_pair, ctx->ntask_group);
  for (int k = 0; k < CQG_NQC; ++k) {
    int i, j;
    qclass_split(k, i, j);
    ctx->class_possible[k] = ctx->pc_beg[i + 1] > ctx->pc_beg[i] && ctx->pc_beg[j + 1] > ctx->pc_beg[j];
  }
  size_t scan_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (long long *)nullptr, (long long *)nullptr,
                                std::max(kListParts * task, 1));
  if (ctx->d_cnt.reserve(kListParts * (size_t)task + 1) || ctx->d_off.reserve(kListParts * (size_t)task + 1) ||
      ctx->d_range.reserve(2 * CQG_NLIST) || ctx->d_qhead.reserve(CQG_NLIST + 1) ||
      ctx->d_scan_tmp.reserve(scan_bytes + 16) || ctx->d_M.reserve(2 * (size_t)std::max(ctx->Mtotal, 1LL)) ||
      ctx->d_Mmax.reserve(1) || ctx->d_flags.reserve(4) || ctx->d_blkacc.reserve(kBlkAcc * CQG_NQC) ||
      ctx->d_Mpair.reserve(std::max<size_t>(ctx->pair_sh.size(), 1)))
    return CQG_ERR_OOM;
  return CQG_OK;
}

cqg_status cqg_set_basis(cqg_ctx *ctx, int nshell, const int *L, const int *pure, const int *nprim,
                         const double *alpha, const double *coef, const double *centers) {
  return cqg_set_basis_batch(ctx, 1, &nshell, L, pure, nprim, alpha, coef, centers);
}

cqg_status cqg_get_schwarz(cqg_ctx *ctx, double *Q) {
  if (!ctx || !Q) return CQG_ERR_BAD_ARG;
  if (ctx->nshell == 0) return CQG_ERR_STATE;
  memcpy(Q, ctx->Qmat.data(), ctx->Qmat.size() * sizeof(double));
  return CQG_OK;
}

// Whether quartet class k goes through the class-fused kernel of `tier` (0: none).
// whether work list vb (part * CQG_NQC + class) goes through the class-fused kernel of
// `tier` (the pair entries of the tier's classes; a class index k < CQG_NQC is its FP64 list)
static bool class_fused(int tier, int vb) {
  if (tier == 0 || vb >= 2 * CQG_NQC) return false;
  const int k = vb % CQG_NQC;
  int i, j;
  qclass_split(k, i, j);
  return cqg_fused_member(tier, kPairClass[i][0], kPairClass[i][1], kPairClass[j][0], kPairClass[j][1]);
}

// Launch-shape autotuner: for every (precision, class) list with work, time each candidate
// shape (persistent CTAs per SM; warps per CTA for the warp-cooperative classes) with the
// digest pointed at scratch accumulators, and keep the fastest.
static cqg_status autotune_shapes(cqg_ctx *ctx, const long long *crange, cudaStream_t st, const DigestGroups &dg) {
  DigestGroups scratch = dg;
  size_t per = 0;
  for (int g = 0; g < dg.ng; ++g) per = std::max<size_t>(per, 1);
  const size_t gsize = ctx->nmol > 1 ? (size_t)ctx->packed : (size_t)ctx->nbf * ctx->nbf;
  if (ctx->d_Gscratch.reserve(gsize) != cudaSuccess) return CQG_ERR_OOM;
  for (int g = 0; g < dg.ng; ++g) scratch.G[g] = ctx->d_Gscratch.p;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  for (int vb = 0; vb < CQG_NLIST; ++vb) {
    const long long n = crange[2 * vb + 1] - crange[2 * vb];
    if (n <= 0 || !list_launcher(vb)) continue;
    const int k = vb % CQG_NQC;
    const bool sibling = vb >= 2 * CQG_NQC;
    int i, j;
    qclass_split(k, i, j);
    const int la = kPairClass[i][0], lb = kPairClass[i][1], lc = kPairClass[j][0], ld = kPairClass[j][1];
    const bool warp = !sibling && is_warp_class(la, lb, lc, ld);
    const bool both = !sibling && is_variant_class(la, lb, lc, ld);
    struct Shape {
      int cta, wpb, qpw, var;
    };
    // (CTAs per SM, warps per CTA, quartets claimed per warp, kernel form)
    std::vector<Shape> cand;
    if (sibling) {   // sibling lists: also CTAs of 64 threads (2 warps)
      for (int w : {2, 4})
        for (int c : {4, 8, 16})
          for (int q : {1, 4}) cand.push_back({c, w, q, 0});
    } else if (!warp) {
      for (int c : {4, 8, 12, 16, 24})
        for (int q : {1, 4}) cand.push_back({c, 0, q, 0});
    }
    if (warp || both) {
      for (int w : {1, 2, 4})
        for (int c : {8, 16, 32})
          for (int q : {1, 4}) cand.push_back({c, w, q, warp ? 0 : 1});
    }
    // Long lists are timed on their first quarter (at least 2^20 quartets), after one
    // untimed run, one run per candidate; short lists in full, best of two runs.  The
    // kernels read their range from d_range, so the sample range is written there and the
    // full range put back afterwards.
    const long long m = n > (1ll << 20) ? std::max<long long>(1ll << 20, n / 4) : n;
    const int reps = m < n ? 1 : 2;
    if (m < n) {
      const long long sub[2] = {crange[2 * vb], crange[2 * vb] + m};
      CUCHK(cudaMemcpyAsync(ctx->d_range.p + 2 * vb, sub, sizeof(sub), cudaMemcpyHostToDevice, st));
    }
    float best = 1e30f;
    Shape pick = cand[0];
    for (int ci = (m < n ? -1 : 0); ci < (int)cand.size(); ++ci) {
      const Shape cw = cand[ci < 0 ? 0 : ci];
      ctx->shape_cta[vb] = cw.cta;
      ctx->shape_wpb[vb] = cw.wpb;
      ctx->shape_qpw[vb] = cw.qpw;
      ctx->shape_var[vb] = cw.var;
      float tbest = 1e30f;
      for (int rep = 0; rep < (ci < 0 ? 1 : reps); ++rep) {
        CUCHK(cudaMemsetAsync(ctx->d_qhead.p + vb, 0, sizeof(unsigned long long), st));
        cudaEventRecord(e0, st);
        cudaError_t e = list_launcher(vb)(ctx, vb, m, st, scratch);
        cudaEventRecord(e1, st);
        if (e != cudaSuccess) {
          cudaEventDestroy(e0);
          cudaEventDestroy(e1);
          ctx->err = std::string("autotune launch: ") + cudaGetErrorString(e);
          return CQG_ERR_CUDA;
        }
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        tbest = std::min(tbest, ms);
      }
      if (ci >= 0 && tbest < best) {
        best = tbest;
        pick = cw;
      }
    }
    if (m < n) CUCHK(cudaMemcpyAsync(ctx->d_range.p + 2 * vb, crange + 2 * vb, 2 * sizeof(long long),
                                     cudaMemcpyHostToDevice, st));
    ctx->shape_cta[vb] = pick.cta;
    ctx->shape_wpb[vb] = pick.wpb;
    ctx->shape_qpw[vb] = pick.qpw;
    ctx->shape_var[vb] = pick.var;
  }
  // Class fusion: the lists of the tier-2 classes (every per-thread class up to (dd|dd)) as
  // one launch per list with the shapes just tuned, as the tier-1 fused kernel plus per-list
  // launches of the rest, and as the tier-2 fused kernel; full lists, each timed after one
  // untimed run; the fastest is kept.
  bool any = false;
  for (int vb = 0; vb < CQG_NLIST; ++vb)
    if (crange[2 * vb + 1] > crange[2 * vb] && class_fused(2, vb)) any = true;
  if (any) {
    float best = 1e30f;
    int pick = 0;
    for (int tier = 0; tier <= 2; ++tier) {
      float t = 1e30f;
      for (int rep = 0; rep < 2; ++rep) {
        CUCHK(cudaMemsetAsync(ctx->d_qhead.p, 0, CQG_NLIST * sizeof(unsigned long long), st));
        cudaEventRecord(e0, st);
        cudaError_t e = tier ? cqg_launch_fused(ctx, tier, st, scratch) : cudaSuccess;
        for (int vb = 0; vb < CQG_NLIST && e == cudaSuccess; ++vb) {
          const long long n = crange[2 * vb + 1] - crange[2 * vb];
          if (n <= 0 || !class_fused(2, vb) || class_fused(tier, vb)) continue;
          e = list_launcher(vb)(ctx, vb, n, st, scratch);
        }
        cudaEventRecord(e1, st);
        if (e != cudaSuccess) {
          cudaEventDestroy(e0);
          cudaEventDestroy(e1);
          ctx->err = std::string("autotune (class fusion): ") + cudaGetErrorString(e);
          return CQG_ERR_CUDA;
        }
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep == 1) t = ms;
      }
      ctx->fusion_ms[tier] = t;
      if (t < best) {
        best = t;
        pick = tier;
      }
    }
    ctx->fused_tier = pick;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return CQG_OK;
}

// Sync-free contraction for CUDA-graph capture: the quartet list has a fixed capacity,
// every class kernel reads its range from device memory and runs a persistent grid, and
// nothing is read back.  Overflow of the capacity and invalid inputs are reported through
// device flags (cqg_graph_status).
static cqg_status contract_graph(cqg_ctx *ctx, int ngroups, const double *const *Xg, double *const *AXg,
                                 const double *sJ, const double *sK, int nx_all, const double *const *Xall, int ldx,
                                 int ldax, cudaStream_t st) {
  const Mols mols = make_mols(ctx);
  const size_t gsize = ctx->nmol > 1 ? (size_t)ctx->packed : (size_t)ctx->nbf * ctx->nbf;
  if ((size_t)ngroups * gsize > ctx->d_G.n || (size_t)ctx->graph_capacity > ctx->d_qlist.n ||
      (size_t)ctx->graph_capacity > ctx->d_qmask.n) {
    ctx->err = "graph mode: buffers were not reserved for this call (cqg_set_graph_mode)";
    return CQG_ERR_STATE;
  }
  XList xl;
  xl.n = nx_all;
  for (int i = 0; i < nx_all; ++i) xl.X[i] = Xall[i];
  const double cut32 = ctx->policy == CQG_PREC_MIXED ? ctx->fp32_cutoff : 0.0;
  CUCHK(cudaMemsetAsync(ctx->d_flags.p, 0, 4 * sizeof(int), st));
  CUCHK(cudaMemsetAsync(ctx->d_Mmax.p, 0, sizeof(double), st));
  CUCHK(cudaMemsetAsync(ctx->d_blkacc.p, 0, kBlkAcc * CQG_NQC * sizeof(unsigned long long), st));
  CUCHK(cudaMemsetAsync(ctx->d_mhead.p, 0, sizeof(unsigned long long), st));
  CUCHK(cudaMemsetAsync(ctx->d_G.p, 0, (size_t)ngroups * gsize * sizeof(double), st));
  {
    dim3 g((ctx->max_nsh + 127) / 128, ctx->max_nsh, ctx->nmol);
    k_blocknorm<<<g, 128, 0, st>>>(xl, ldx, mols, ctx->d_bf.p, ctx->d_sz.p, ctx->d_M.p, ctx->d_M.p + ctx->Mtotal, ctx->d_flags.p, 1e-12);
    const long long nn = ctx->Mtotal;
    k_maxreduce<<<(int)std::min<long long>((nn + 255) / 256, 1184), 256, 0, st>>>(ctx->d_M.p, nn, ctx->d_Mmax.p);
    const int npairs = (int)ctx->pair_sh.size();
    k_pairnorm<<<(npairs + 255) / 256, 256, 0, st>>>(ctx->d_pair_sh.p, npairs, mols, ctx->d_shmol.p, ctx->d_M.p,
                                                     ctx->d_Mpair.p);
  }
  Pairs P = make_pairs(ctx);
  const int nb = (ctx->ntask + 7) / 8;
  k_quartets<false><<<nb, 256, 0, st>>>(ctx->bt, ctx->ntask, P, ctx->d_M.p, ctx->d_M.p + ctx->Mtotal, ctx->d_Mpair.p, mols, ctx->d_shmol.p, ctx->d_Mmax.p,
                                         ctx->thresh, cut32, ctx->d_cnt.p, nullptr, nullptr, nullptr, ctx->d_blkacc.p,
                                         0, 0, 0, 0, make_mask_cache(ctx));
  size_t scan_bytes = ctx->d_scan_tmp.n;
  CUCHK(cub::DeviceScan::ExclusiveSum(ctx->d_scan_tmp.p, scan_bytes, ctx->d_cnt.p, ctx->d_off.p,
                                      kListParts * ctx->ntask, st));
  k_block_ranges<<<1, kRangeThreads, 0, st>>>(ctx->bt, ctx->ntask, ctx->d_cnt.p, ctx->d_off.p, ctx->d_range.p,
                                    ctx->graph_capacity, ctx->d_flags.p);
  k_quartets<true><<<nb, 256, 0, st>>>(ctx->bt, ctx->ntask, P, ctx->d_M.p, ctx->d_M.p + ctx->Mtotal, ctx->d_Mpair.p, mols, ctx->d_shmol.p, ctx->d_Mmax.p,
                                        ctx->thresh, cut32, nullptr, ctx->d_off.p, ctx->d_qlist.p, ctx->d_qmask.p,
                                        nullptr, 0,
                                        (long long)kListParts * ctx->ntask, 0, ctx->graph_capacity,
                                        make_mask_cache(ctx));
  CUCHK(cudaGetLastError());
  DigestGroups dg;
  memset(&dg, 0, sizeof(dg));
  dg.ng = ngroups;
  dg.ldx = ldx;
  dg.batch = ctx->nmol > 1;
  dg.xoff = ctx->d_mxoff.p;
  dg.nbf = ctx->d_mnbf.p;
  for (int g = 0; g < ngroups; ++g) {
    dg.X[g] = Xg[g];
    dg.G[g] = ctx->d_G.p + (size_t)g * gsize;
    dg.sJ[g] = sJ[g];
    dg.sK[g] = sK[g];
  }
  CUCHK(cudaMemsetAsync(ctx->d_qhead.p, 0, CQG_NLIST * sizeof(unsigned long long), st));
  int launches = 7;   // block norms, max, pair norms, list count, scan, ranges, list fill
  if (ctx->fused_tier) {
    cudaError_t e = cqg_launch_fused(ctx, ctx->fused_tier, st, dg);
    ++launches;
    if (e != cudaSuccess) {
      ctx->err = std::string("class-fused eri kernel: ") + cudaGetErrorString(e);
      return CQG_ERR_CUDA;
    }
  }
  for (int vb = 0; vb < CQG_NLIST; ++vb) {
    const int k = vb % CQG_NQC, part = vb / CQG_NQC;
    if (!ctx->class_possible[k] || class_fused(ctx->fused_tier, vb) || !list_launcher(vb)) continue;
    if ((part & 1) && ctx->policy != CQG_PREC_MIXED) continue;   // FP32 lists are empty
    if (part >= 2 && !ctx->bt.grouped[k]) continue;               // no sibling entries
    cudaError_t e = list_launcher(vb)(ctx, vb, -1, st, dg);
    ++launches;
    if (e != cudaSuccess) {
      ctx->err = std::string("eri kernel ") + cqg_class_name(k) + ": " + cudaGetErrorString(e);
      return CQG_ERR_CUDA;
    }
  }
  for (int g = 0; g < ngroups; ++g) {
    dim3 grid((ctx->max_nbf + 31) / 32, (ctx->max_nbf + 31) / 32, ctx->nmol), blk(32, 8);
    k_finalize<<<grid, blk, 0, st>>>(dg.G[g], mols, AXg[g], ldax);
    ++launches;
  }
  CUCHK(cudaGetLastError());
  ctx->launches = launches;
  ctx->stats.launches = launches;
  return CQG_OK;
}

static cqg_status contract_device(cqg_ctx *ctx, int ngroups, const double *const *Xg, double *const *AXg,
                                  const double *sJ, const double *sK, int nx_all, const double *const *Xall,
                                  int ldx, int ldax, cudaStream_t st) {
  const int n = ctx->nbf;
  const Mols mols = make_mols(ctx);
  // Gh of every molecule: n x n for one molecule, packed per molecule for a batch
  const size_t gsize = ctx->nmol > 1 ? (size_t)ctx->packed : (size_t)n * n;
  // the survivor-mask cache: grow it to what the last count pass asked for (tasks that did
  // not fit tested their bounds twice), before this call's first launch; never in graph
  // mode, whose captured launches hold the buffer's address
  if (ctx->graph_capacity == 0 && ctx->mask_steps_used > (long long)ctx->d_masks.n) {
    const long long want = std::min<long long>(ctx->mask_steps_used + ctx->mask_steps_used / 4, kMaskStepsMax);
    if (want > (long long)ctx->d_masks.n && ctx->d_masks.reserve((size_t)want) != cudaSuccess &&
        ctx->d_masks.reserve((size_t)kMaskStepsInitial) != cudaSuccess) {
      ctx->err = "survivor-mask cache allocation failed";
      return CQG_ERR_OOM;
    }
  }
  if (ctx->timing) CUCHK(cudaEventRecord(ctx->ev[0], st));
  // 1. block norms + checks
  XList xl;
  xl.n = nx_all;
  for (int i = 0; i < nx_all; ++i) xl.X[i] = Xall[i];
  CUCHK(cudaMemsetAsync(ctx->d_flags.p, 0, 4 * sizeof(int), st));
  CUCHK(cudaMemsetAsync(ctx->d_Mmax.p, 0, sizeof(double), st));
  CUCHK(cudaMemsetAsync(ctx->d_blkacc.p, 0, kBlkAcc * CQG_NQC * sizeof(unsigned long long), st));
  CUCHK(cudaMemsetAsync(ctx->d_mhead.p, 0, sizeof(unsigned long long), st));
  const double cut32 = ctx->policy == CQG_PREC_MIXED ? ctx->fp32_cutoff : 0.0;
  ctx->launches = 0;
  {
    dim3 g((ctx->max_nsh + 127) / 128, ctx->max_nsh, ctx->nmol);
    k_blocknorm<<<g, 128, 0, st>>>(xl, ldx, mols, ctx->d_bf.p, ctx->d_sz.p, ctx->d_M.p, ctx->d_M.p + ctx->Mtotal, ctx->d_flags.p, 1e-12);
    CUCHK(cudaGetLastError());
    long long nn = ctx->Mtotal;
    int nb = (int)std::min<long long>((nn + 255) / 256, 1184);
    k_maxreduce<<<nb, 256, 0, st>>>(ctx->d_M.p, nn, ctx->d_Mmax.p);
    const int npairs = (int)ctx->pair_sh.size();
    k_pairnorm<<<(npairs + 255) / 256, 256, 0, st>>>(ctx->d_pair_sh.p, npairs, mols, ctx->d_shmol.p, ctx->d_M.p,
                                                     ctx->d_Mpair.p);
    CUCHK(cudaGetLastError());
    ctx->launches += 3;
  }
  // 2. quartet lists
  Pairs P = make_pairs(ctx);
  {
    int nthr = 256, wpb = nthr / 32;
    int nb = (ctx->ntask + wpb - 1) / wpb;
    k_quartets<false><<<nb, nthr, 0, st>>>(ctx->bt, ctx->ntask, P, ctx->d_M.p, ctx->d_M.p + ctx->Mtotal, ctx->d_Mpair.p, mols, ctx->d_shmol.p, ctx->d_Mmax.p,
                                            ctx->thresh,
                                            cut32, ctx->d_cnt.p, nullptr, nullptr, nullptr, ctx->d_blkacc.p, 0, 0, 0,
                                            0, make_mask_cache(ctx));
    CUCHK(cudaGetLastError());
    size_t scan_bytes = ctx->d_scan_tmp.n;
    CUCHK(cub::DeviceScan::ExclusiveSum(ctx->d_scan_tmp.p, scan_bytes, ctx->d_cnt.p, ctx->d_off.p,
                                      kListParts * ctx->ntask, st));
    k_block_ranges<<<1, kRangeThreads, 0, st>>>(ctx->bt, ctx->ntask, ctx->d_cnt.p, ctx->d_off.p, ctx->d_range.p, LLONG_MAX,
                                      ctx->d_flags.p);
    CUCHK(cudaGetLastError());
    ctx->launches += 2;
  }
  long long hr[2 * CQG_NLIST];
  unsigned long long hacc[kBlkAcc * CQG_NQC];
  int hflags[4];
  CUCHK(cudaMemcpyAsync(hr, ctx->d_range.p, sizeof(hr), cudaMemcpyDeviceToHost, st));
  CUCHK(cudaMemcpyAsync(hacc, ctx->d_blkacc.p, sizeof(hacc), cudaMemcpyDeviceToHost, st));
  CUCHK(cudaMemcpyAsync(hflags, ctx->d_flags.p, sizeof(hflags), cudaMemcpyDeviceToHost, st));
  unsigned long long hsteps = 0;
  CUCHK(cudaMemcpyAsync(&hsteps, ctx->d_mhead.p, sizeof(hsteps), cudaMemcpyDeviceToHost, st));
  CUCHK(cudaStreamSynchronize(st));
  ctx->mask_steps_used = (long long)hsteps;
  if (hflags[0]) {
    ctx->err = "input density contains NaN or Inf";
    return CQG_ERR_NONFINITE;
  }
  if (hflags[1]) {
    ctx->err = "input matrix is not symmetric; this engine contracts real symmetric X only";
    return CQG_ERR_UNSUPPORTED;
  }
  long long total = hr[2 * CQG_NLIST - 1];
  // The list is [FP64 pair entries of every task][FP32 pair entries][FP64 sibling
  // entries][FP32 sibling entries] ("virtual tasks" 0 .. 4 ntask).  It is filled and
  // consumed in chunks of at most `list_budget` entries.
  const long long budget = std::max<long long>(ctx->list_budget, 1);
  std::vector<long long> chunk_vt;   // chunk boundaries in virtual tasks
  std::vector<long long> hoff, hcnt;
  const long long nvt = (long long)kListParts * ctx->ntask;
  if (total <= budget) {
    chunk_vt = {0, nvt};
  } else {
    hoff.resize(nvt);
    hcnt.resize(nvt);
    CUCHK(cudaMemcpyAsync(hoff.data(), ctx->d_off.p, nvt * sizeof(long long), cudaMemcpyDeviceToHost, st));
    CUCHK(cudaMemcpyAsync(hcnt.data(), ctx->d_cnt.p, nvt * sizeof(long long), cudaMemcpyDeviceToHost, st));
    CUCHK(cudaStreamSynchronize(st));
    chunk_vt.push_back(0);
    long long start = 0;
    for (long long v = 0; v < nvt; ++v) {
      if (hoff[v] + hcnt[v] - start > budget && v > chunk_vt.back()) {
        chunk_vt.push_back(v);
        start = hoff[v];
      }
    }
    chunk_vt.push_back(nvt);
  }
  long long cap = std::min(total, budget);
  if (chunk_vt.size() > 2) {   // a single task may exceed the budget: size to the largest chunk
    cap = 0;
    for (size_t c = 0; c + 1 < chunk_vt.size(); ++c) {
      const long long v0 = chunk_vt[c], v1 = chunk_vt[c + 1];
      cap = std::max(cap, hoff[v1 - 1] + hcnt[v1 - 1] - hoff[v0]);
    }
  }
  if (ctx->d_qlist.reserve((size_t)std::max<long long>(cap, 1)) != cudaSuccess ||
      ctx->d_qmask.reserve((size_t)std::max<long long>(cap, 1)) != cudaSuccess) {
    ctx->err = "quartet list allocation failed";
    return CQG_ERR_OOM;
  }
  ctx->stats.chunks = (long long)chunk_vt.size() - 1;
  if (ctx->d_G.reserve((size_t)ngroups * gsize) != cudaSuccess) return CQG_ERR_OOM;
  CUCHK(cudaMemsetAsync(ctx->d_G.p, 0, (size_t)ngroups * gsize * sizeof(double), st));
  DigestGroups dg;
  memset(&dg, 0, sizeof(dg));
  dg.ng = ngroups;
  dg.ldx = ldx;
  dg.batch = ctx->nmol > 1;
  dg.xoff = ctx->d_mxoff.p;
  dg.nbf = ctx->d_mnbf.p;
  for (int g = 0; g < ngroups; ++g) {
    dg.X[g] = Xg[g];
    dg.G[g] = ctx->d_G.p + (size_t)g * gsize;
    dg.sJ[g] = sJ[g];
    dg.sK[g] = sK[g];
  }
  memset(ctx->stats.class_quartets, 0, sizeof(ctx->stats.class_quartets));
  memset(ctx->stats.class_ms, 0, sizeof(ctx->stats.class_ms));
  ctx->stats.ms_fused = 0.0;
  ctx->stats.fused_tier = ctx->fused_tier;
  double mflops = 0, mflops32 = 0;
  long long nprimq = 0, nq32 = 0, nquart = 0;
  for (int k = 0; k < CQG_NQC; ++k) {
    // contracted quartets (a sibling-group entry of the list holds several)
    const int b = k;
    const long long n64 = (long long)hacc[kBlkAcc * b + 4];
    const long long n32 = (long long)hacc[kBlkAcc * b + 5];
    ctx->stats.class_quartets[k] += n64 + n32;
    nq32 += n32;
    nquart += n64 + n32;
    int i, j;
    qclass_split(k, i, j);
    const int la = kPairClass[i][0], lb = kPairClass[i][1], lc = kPairClass[j][0], ld = kPairClass[j][1];
    const double fp = md_v1_prim_flops(la, lb, lc, ld), fd = md_v1_digest_flops(la, lb, lc, ld);
    mflops += (double)hacc[kBlkAcc * b] * fp + (double)n64 * fd;
    mflops32 += (double)hacc[kBlkAcc * b + 2] * fp + (double)n32 * fd;
    nprimq += (long long)(hacc[kBlkAcc * b + 1] + hacc[kBlkAcc * b + 3]);
  }
  bool first_chunk = true;
  bool timed[CQG_NQC] = {false};
  for (size_t ch = 0; ch + 1 < chunk_vt.size(); ++ch) {
    const long long vt0 = chunk_vt[ch], vt1 = chunk_vt[ch + 1];
    long long obase = 0;
    long long crange[2 * CQG_NLIST];
    if (chunk_vt.size() > 2) {
      obase = hoff[vt0];
      for (int vb = 0; vb < CQG_NLIST; ++vb) {
        const int prec = vb / CQG_NQC, b = vb % CQG_NQC;
        long long t0 = (long long)prec * ctx->ntask + ctx->bt.task_beg[b];
        long long t1 = (long long)prec * ctx->ntask + ctx->bt.task_beg[b + 1];
        t0 = std::max(t0, vt0);
        t1 = std::min(t1, vt1);
        if (t1 > t0) {
          crange[2 * vb] = hoff[t0] - obase;
          crange[2 * vb + 1] = hoff[t1 - 1] + hcnt[t1 - 1] - obase;
        } else {
          crange[2 * vb] = crange[2 * vb + 1] = 0;
        }
      }
      CUCHK(cudaMemcpyAsync(ctx->d_range.p, crange, sizeof(crange), cudaMemcpyHostToDevice, st));
    } else {
      for (int q = 0; q < 2 * CQG_NLIST; ++q) crange[q] = hr[q];
    }
    {
      int nthr = 256, wpb = nthr / 32;
      int nb = (ctx->ntask + wpb - 1) / wpb;
      k_quartets<true><<<nb, nthr, 0, st>>>(ctx->bt, ctx->ntask, P, ctx->d_M.p, ctx->d_M.p + ctx->Mtotal, ctx->d_Mpair.p, mols, ctx->d_shmol.p, ctx->d_Mmax.p,
                                             ctx->thresh,
                                             cut32, nullptr, ctx->d_off.p, ctx->d_qlist.p, ctx->d_qmask.p, nullptr,
                                             vt0, vt1, obase,
                                             (long long)std::min(ctx->d_qlist.n, ctx->d_qmask.n),
                                             make_mask_cache(ctx));
      CUCHK(cudaGetLastError());
      ctx->launches += 1;
    }
    if (ctx->timing && first_chunk) CUCHK(cudaEventRecord(ctx->ev[1], st));
    if (ctx->autotune_pending && chunk_vt.size() == 2) {
      cqg_status ts = autotune_shapes(ctx, crange, st, dg);
      if (ts != CQG_OK) return ts;
      ctx->autotune_pending = 0;
    }
    // 3. ERI + digest per class, each list consumed through its work-queue head counter
    CUCHK(cudaMemsetAsync(ctx->d_qhead.p, 0, CQG_NLIST * sizeof(unsigned long long), st));
    if (ctx->fused_tier) {   // the fused tier's lists in one launch (its time: ms_fused)
      if (ctx->timing) CUCHK(cudaEventRecord(ctx->ev[4 + 2 * CQG_NQC], st));
      cudaError_t e = cqg_launch_fused(ctx, ctx->fused_tier, st, dg);
      if (e != cudaSuccess) {
        ctx->err = std::string("class-fused eri kernel: ") + cudaGetErrorString(e);
        return CQG_ERR_CUDA;
      }
      if (ctx->timing) CUCHK(cudaEventRecord(ctx->ev[5 + 2 * CQG_NQC], st));
      ctx->launches += 1;
    }
    for (int k = 0; k < CQG_NQC; ++k) {   // the class's lists: pair entries FP64, FP32, sibling entries FP64, FP32
      bool any_list = false;
      for (int part = 0; part < kListParts; ++part) {
        const int vb = part * CQG_NQC + k;
        if (!class_fused(ctx->fused_tier, vb) && crange[2 * vb + 1] > crange[2 * vb]) any_list = true;
      }
      if (!any_list) continue;
      if (ctx->timing) CUCHK(cudaEventRecord(ctx->ev[4 + 2 * k], st));
      for (int part = 0; part < kListParts; ++part) {
        const int vb = part * CQG_NQC + k;
        const long long n = crange[2 * vb + 1] - crange[2 * vb];
        if (n <= 0 || class_fused(ctx->fused_tier, vb)) continue;
        if (!list_launcher(vb)) {
          ctx->err = std::string("sibling entries for a class without the sibling form: ") + cqg_class_name(k);
          return CQG_ERR_STATE;
        }
        ctx->launches += 1;
        cudaError_t e = list_launcher(vb)(ctx, vb, n, st, dg);
        if (e != cudaSuccess) {
          ctx->err = std::string("eri kernel ") + cqg_class_name(k) + ": " + cudaGetErrorString(e);
          return CQG_ERR_CUDA;
        }
      }
      if (ctx->timing) {
        CUCHK(cudaEventRecord(ctx->ev[5 + 2 * k], st));
        timed[k] = true;
      }
    }
    if (ctx->timing) {   // per-class device time (all lists of the class), summed over chunks
      CUCHK(cudaStreamSynchronize(st));
      for (int k = 0; k < CQG_NQC; ++k) {
        float ms = 0.f;
        if (timed[k] && cudaEventElapsedTime(&ms, ctx->ev[4 + 2 * k], ctx->ev[5 + 2 * k]) == cudaSuccess)
          ctx->stats.class_ms[k] += ms;
        timed[k] = false;
      }
      float ms = 0.f;
      if (ctx->fused_tier &&
          cudaEventElapsedTime(&ms, ctx->ev[4 + 2 * CQG_NQC], ctx->ev[5 + 2 * CQG_NQC]) == cudaSuccess)
        ctx->stats.ms_fused += ms;
    }
    first_chunk = false;
  }
  if (ctx->timing) CUCHK(cudaEventRecord(ctx->ev[2], st));
  // 4. AX += 0.5 (Gh + Gh^T)
  for (int g = 0; g < ngroups; ++g) {
    dim3 grid((ctx->max_nbf + 31) / 32, (ctx->max_nbf + 31) / 32, ctx->nmol), blk(32, 8);
    k_finalize<<<grid, blk, 0, st>>>(dg.G[g], mols, AXg[g], ldax);
    CUCHK(cudaGetLastError());
    ctx->launches += 1;
  }
  if (ctx->timing) CUCHK(cudaEventRecord(ctx->ev[3], st));
  ctx->stats.quartets = nquart;
  ctx->stats.list_entries = total;
  ctx->stats.sibling_classes = 0;
  for (int k = 0; k < CQG_NQC; ++k) {   // classes whose sibling-group lists had entries
    const int v64 = 2 * CQG_NQC + k, v32 = 3 * CQG_NQC + k;
    if (hr[2 * v64 + 1] > hr[2 * v64] || hr[2 * v32 + 1] > hr[2 * v32]) ctx->stats.sibling_classes |= 1LL << k;
  }
  ctx->stats.quartets_fp32 = nq32;
  ctx->stats.model_flops = mflops + mflops32;
  ctx->stats.model_flops_fp32 = mflops32;
  ctx->stats.prim_quartets = nprimq;
  ctx->stats.launches = ctx->launches;
  return CQG_OK;
}

// group (X, AX) pairs and fold scales: COULOMB -> sJ, EXCHANGE -> sK
static cqg_status plan_groups(cqg_ctx *ctx, int nmat, const double *const *X, double *const *AX, const int *types,
                              const double *scale, int &ng, const double **Xg, double **AXg, double *sJ, double *sK,
                              int &nxu, const double **Xu) {
  ng = 0;
  nxu = 0;
  for (int i = 0; i < nmat; ++i) {
    if (!X[i] || !AX[i] || (types[i] != CQG_COULOMB && types[i] != CQG_EXCHANGE)) {
      ctx->err = "null matrix or unknown contraction type";
      return CQG_ERR_BAD_ARG;
    }
    bool seen = false;
    for (int u = 0; u < nxu; ++u)
      if (Xu[u] == X[i]) seen = true;
    if (!seen) {
      if (nxu >= 8) return CQG_ERR_BAD_ARG;
      Xu[nxu++] = X[i];
    }
    int g = -1;
    for (int k = 0; k < ng; ++k)
      if (Xg[k] == X[i] && AXg[k] == AX[i]) g = k;
    if (g < 0) {
      if (ng >= CQG_MAXG) {
        ctx->err = "too many distinct (X, AX) pairs in one call";
        return CQG_ERR_UNSUPPORTED;
      }
      g = ng++;
      Xg[g] = X[i];
      AXg[g] = AX[i];
      sJ[g] = sK[g] = 0.0;
    }
    if (types[i] == CQG_COULOMB) sJ[g] += scale[i];
    else sK[g] += scale[i];
  }
  return CQG_OK;
}

cqg_status cqg_twoe_contract_direct(cqg_ctx *ctx, int nmat, const double *const *X, double *const *AX,
                                    const int *types, const double *scale, int ld, int on_device, void *stream) {
  if (!ctx) return CQG_ERR_BAD_ARG;
  if (ctx->nshell == 0) {
    ctx->err = "cqg_set_basis has not been called";
    return CQG_ERR_STATE;
  }
  if (nmat <= 0 || nmat > 8 || !X || !AX || !types || !scale || ld < ctx->nbf) {
    ctx->err = "bad list sizes or leading dimension";
    return CQG_ERR_BAD_ARG;
  }
  CUCHK(cudaSetDevice(ctx->device));
  cudaStream_t st = (cudaStream_t)stream;
  const double *Xg[CQG_MAXG];
  double *AXg[CQG_MAXG];
  double sJ[CQG_MAXG], sK[CQG_MAXG];
  const double *Xu[8];
  int ng, nxu;
  cqg_status s = plan_groups(ctx, nmat, X, AX, types, scale, ng, Xg, AXg, sJ, sK, nxu, Xu);
  if (s != CQG_OK) return s;
  const int n = ctx->nbf;
  if (on_device && ctx->graph_capacity > 0) return contract_graph(ctx, ng, Xg, AXg, sJ, sK, nxu, Xu, ld, ld, st);
  if (on_device) return contract_device(ctx, ng, Xg, AXg, sJ, sK, nxu, Xu, ld, ld, st);
  // host pointers: stage distinct X and each group's AX on the device
  size_t nn = (size_t)n * n;
  if (ctx->d_X.reserve(nn * nxu) || ctx->d_AX.reserve(nn * ng)) return CQG_ERR_OOM;
  const double *dXu[8];
  for (int u = 0; u < nxu; ++u) {
    dXu[u] = ctx->d_X.p + nn * u;
    CUCHK(cudaMemcpy2DAsync((void *)dXu[u], n * sizeof(double), Xu[u], ld * sizeof(double), n * sizeof(double), n,
                            cudaMemcpyHostToDevice, st));
  }
  const double *dXg[CQG_MAXG];
  double *dAXg[CQG_MAXG];
  for (int g = 0; g < ng; ++g) {
    for (int u = 0; u < nxu; ++u)
      if (Xu[u] == Xg[g]) dXg[g] = dXu[u];
    dAXg[g] = ctx->d_AX.p + nn * g;
    CUCHK(cudaMemcpy2DAsync(dAXg[g], n * sizeof(double), AXg[g], ld * sizeof(double), n * sizeof(double), n,
                            cudaMemcpyHostToDevice, st));
  }
  s = contract_device(ctx, ng, dXg, dAXg, sJ, sK, nxu, dXu, n, n, st);
  if (s != CQG_OK) return s;
  for (int g = 0; g < ng; ++g)
    CUCHK(cudaMemcpy2DAsync(AXg[g], ld * sizeof(double), dAXg[g], n * sizeof(double), n * sizeof(double), n,
                            cudaMemcpyDeviceToHost, st));
  CUCHK(cudaStreamSynchronize(st));
  return CQG_OK;
}

cqg_status cqg_form_pt(cqg_ctx *ctx, int is_rhf, double xHF, const double *Ps, const double *Pz, double *PTs,
                       double *PTz, int ld, int on_device, void *stream) {
  if (!ctx || !Ps || !PTs || (!is_rhf && (!Pz || !PTz))) return CQG_ERR_BAD_ARG;
  if (ctx->nshell == 0) {
    ctx->err = "cqg_set_basis has not been called";
    return CQG_ERR_STATE;
  }
  const int n = ctx->nbf;
  if (ld < n) {   // checked before PT is zeroed: nothing is written on a bad call
    ctx->err = "leading dimension below the number of basis functions";
    return CQG_ERR_BAD_ARG;
  }
  CUCHK(cudaSetDevice(ctx->device));
  cudaStream_t st = (cudaStream_t)stream;
  // PT zeroed first (singleslater_fock.h:47,54)
  if (on_device) {
    CUCHK(cudaMemset2DAsync(PTs, ld * sizeof(double), 0, n * sizeof(double), n, st));
    if (!is_rhf) CUCHK(cudaMemset2DAsync(PTz, ld * sizeof(double), 0, n * sizeof(double), n, st));
  } else {
    for (int c = 0; c < n; ++c) memset(PTs + (size_t)c * ld, 0, n * sizeof(double));
    if (!is_rhf)
      for (int c = 0; c < n; ++c) memset(PTz + (size_t)c * ld, 0, n * sizeof(double));
  }
  if (is_rhf) {
    const double *X[2] = {Ps, Ps};
    double *AX[2] = {PTs, PTs};
    int types[2] = {CQG_COULOMB, CQG_EXCHANGE};
    double scale[2] = {1.0, xHF};
    return cqg_twoe_contract_direct(ctx, 2, X, AX, types, scale, ld, on_device, stream);
  }
  const double *X[3] = {Ps, Ps, Pz};
  double *AX[3] = {PTs, PTs, PTz};
  int types[3] = {CQG_COULOMB, CQG_EXCHANGE, CQG_EXCHANGE};
  double scale[3] = {1.0, xHF, xHF};
  return cqg_twoe_contract_direct(ctx, 3, X, AX, types, scale, ld, on_device, stream);
}

cqg_status cqg_one_e(cqg_ctx *ctx, int ncharge, const double *Z, const double *R, double *S, double *T, double *V,
                     int ld, int on_device, void *stream) {
  if (!ctx || ncharge < 0 || (ncharge > 0 && (!Z || !R)) || !S || !T || !V) return CQG_ERR_BAD_ARG;
  if (ctx->nshell == 0) {
    ctx->err = "cqg_set_basis has not been called";
    return CQG_ERR_STATE;
  }
  const int n = ctx->nbf;
  if (ld < n) return CQG_ERR_BAD_ARG;
  CUCHK(cudaSetDevice(ctx->device));
  cudaStream_t st = (cudaStream_t)stream;
  if (ctx->d_charges.reserve(4 * (size_t)std::max(ncharge, 1))) return CQG_ERR_OOM;
  std::vector<double> zr(4 * (size_t)std::max(ncharge, 1), 0.0);
  for (int c = 0; c < ncharge; ++c) {
    zr[c] = Z[c];
    zr[ncharge + 3 * c] = R[3 * c];
    zr[ncharge + 3 * c + 1] = R[3 * c + 1];
    zr[ncharge + 3 * c + 2] = R[3 * c + 2];
  }
  CUCHK(cudaMemcpyAsync(ctx->d_charges.p, zr.data(), zr.size() * sizeof(double), cudaMemcpyHostToDevice, st));
  double *dS = S, *dT = T, *dV = V;
  int ldd = ld;
  if (!on_device) {
    if (ctx->d_oe.reserve(3 * (size_t)n * n)) return CQG_ERR_OOM;
    dS = ctx->d_oe.p;
    dT = dS + (size_t)n * n;
    dV = dT + (size_t)n * n;
    ldd = n;
  }
  OneEShells sh;
  sh.L = ctx->d_shL.p;
  sh.nprim = ctx->d_shnp.p;
  sh.poff = ctx->d_shpoff.p;
  sh.bf = ctx->d_bf.p;
  sh.alpha = ctx->d_alpha.p;
  sh.coef = ctx->d_coef.p;
  sh.center = ctx->d_center.p;
  if (ctx->nmol != 1) {
    ctx->err = "cqg_one_e is for single-molecule contexts; use cqg_one_e_batch";
    return CQG_ERR_STATE;
  }
  const long long np = ctx->nallpairs;
  OneEMols om;
  memset(&om, 0, sizeof(om));
  k_one_e<<<(unsigned)((np + 63) / 64), 64, 0, st>>>(sh, ctx->d_allpairs.p, np, ncharge, ctx->d_charges.p,
                                                     (const double3 *)(ctx->d_charges.p + ncharge), ctx->d_boys.p, dS,
                                                     dT, dV, ldd, om);
  CUCHK(cudaGetLastError());
  if (!on_device) {
    double *outs[3] = {S, T, V};
    const double *ins[3] = {dS, dT, dV};
    for (int q = 0; q < 3; ++q)
      CUCHK(cudaMemcpy2DAsync(outs[q], ld * sizeof(double), ins[q], n * sizeof(double), n * sizeof(double), n,
                              cudaMemcpyDeviceToHost, st));
    CUCHK(cudaStreamSynchronize(st));
  }
  return CQG_OK;
}

cqg_status cqg_dipole(cqg_ctx *ctx, const double *origin, double *D, int ld, int on_device, void *stream) {
  if (!ctx || !origin || !D) return CQG_ERR_BAD_ARG;
  if (ctx->nshell == 0) {
    ctx->err = "cqg_set_basis has not been called";
    return CQG_ERR_STATE;
  }
  if (ctx->nmol != 1) {
    ctx->err = "cqg_dipole is for single-molecule contexts";
    return CQG_ERR_STATE;
  }
  const int n = ctx->nbf;
  if (ld < n) {
    ctx->err = "leading dimension below the number of basis functions";
    return CQG_ERR_BAD_ARG;
  }
  CUCHK(cudaSetDevice(ctx->device));
  cudaStream_t st = (cudaStream_t)stream;
  double *dD = D;
  int ldd = ld;
  if (!on_device) {
    if (ctx->d_oe.reserve(3 * (size_t)n * n)) return CQG_ERR_OOM;
    dD = ctx->d_oe.p;
    ldd = n;
  }
  OneEShells sh;
  sh.L = ctx->d_shL.p;
  sh.nprim = ctx->d_shnp.p;
  sh.poff = ctx->d_shpoff.p;
  sh.bf = ctx->d_bf.p;
  sh.alpha = ctx->d_alpha.p;
  sh.coef = ctx->d_coef.p;
  sh.center = ctx->d_center.p;
  const long long np = ctx->nallpairs;
  k_dipole<<<(unsigned)((np + 63) / 64), 64, 0, st>>>(sh, ctx->d_allpairs.p, np,
                                                      make_double3(origin[0], origin[1], origin[2]), dD, ldd, n);
  CUCHK(cudaGetLastError());
  if (!on_device) {
    for (int k = 0; k < 3; ++k)
      CUCHK(cudaMemcpy2DAsync(D + (size_t)k * ld * n, ld * sizeof(double), dD + (size_t)k * n * n,
                              n * sizeof(double), n * sizeof(double), n, cudaMemcpyDeviceToHost, st));
    CUCHK(cudaStreamSynchronize(st));
  }
  return CQG_OK;
}

cqg_status cqg_one_e_batch(cqg_ctx *ctx, const int *ncharge_per_mol, const double *Z, const double *R, double *S,
                           double *T, double *V, void *stream) {
  if (!ctx || !ncharge_per_mol || !Z || !R || !S || !T || !V) return CQG_ERR_BAD_ARG;
  if (ctx->nshell == 0) return CQG_ERR_STATE;
  CUCHK(cudaSetDevice(ctx->device));
  cudaStream_t st = (cudaStream_t)stream;
  const int nmol = ctx->nmol;
  std::vector<int> coff(nmol + 1, 0);
  for (int m = 0; m < nmol; ++m) coff[m + 1] = coff[m] + ncharge_per_mol[m];
  const int nc = coff[nmol];
  if (ctx->d_charges.reserve(4 * (size_t)std::max(nc, 1) + nmol + 1)) return CQG_ERR_OOM;
  std::vector<double> zr(4 * (size_t)std::max(nc, 1) + nmol + 1, 0.0);
  for (int c = 0; c < nc; ++c) {
    zr[c] = Z[c];
    zr[nc + 3 * c] = R[3 * c];
    zr[nc + 3 * c + 1] = R[3 * c + 1];
    zr[nc + 3 * c + 2] = R[3 * c + 2];
  }
  int *dcoff = (int *)(ctx->d_charges.p + 4 * (size_t)std::max(nc, 1));
  CUCHK(cudaMemcpyAsync(ctx->d_charges.p, zr.data(), 4 * (size_t)std::max(nc, 1) * sizeof(double),
                        cudaMemcpyHostToDevice, st));
  CUCHK(cudaMemcpyAsync(dcoff, coff.data(), (nmol + 1) * sizeof(int), cudaMemcpyHostToDevice, st));
  OneEShells sh;
  sh.L = ctx->d_shL.p;
  sh.nprim = ctx->d_shnp.p;
  sh.poff = ctx->d_shpoff.p;
  sh.bf = ctx->d_bf.p;
  sh.alpha = ctx->d_alpha.p;
  sh.coef = ctx->d_coef.p;
  sh.center = ctx->d_center.p;
  OneEMols om;
  om.shmol = ctx->d_shmol.p;
  om.xoff = ctx->d_mxoff.p;
  om.nbf = ctx->d_mnbf.p;
  om.coff = dcoff;
  om.batch = 1;
  const long long np = ctx->nallpairs;
  k_one_e<<<(unsigned)((np + 63) / 64), 64, 0, st>>>(sh, ctx->d_allpairs.p, np, nc, ctx->d_charges.p,
                                                     (const double3 *)(ctx->d_charges.p + nc), ctx->d_boys.p, S, T,
                                                     V, 0, om);
  CUCHK(cudaGetLastError());
  return CQG_OK;
}

cqg_status cqg_get_batch_layout(cqg_ctx *ctx, int *nbf_per_mol, long long *offset_per_mol, long long *packed) {
  if (!ctx) return CQG_ERR_BAD_ARG;
  for (int m = 0; m < ctx->nmol; ++m) {
    if (nbf_per_mol) nbf_per_mol[m] = ctx->m_nbf[m];
    if (offset_per_mol) offset_per_mol[m] = ctx->m_xoff[m];
  }
  if (packed) *packed = ctx->packed;
  return CQG_OK;
}

cqg_status cqg_twoe_contract_direct_batch(cqg_ctx *ctx, int nmat, const double *const *X, double *const *AX,
                                          const int *types, const double *scale, const unsigned char *active,
                                          void *stream) {
  if (!ctx) return CQG_ERR_BAD_ARG;
  if (ctx->nshell == 0) {
    ctx->err = "cqg_set_basis_batch has not been called";
    return CQG_ERR_STATE;
  }
  if (nmat <= 0 || nmat > 8 || !X || !AX || !types || !scale) return CQG_ERR_BAD_ARG;
  CUCHK(cudaSetDevice(ctx->device));
  cudaStream_t st = (cudaStream_t)stream;
  const unsigned char all1 = 1;
  bool changed = false;
  for (int m = 0; m < ctx->nmol; ++m) {
    const unsigned char a = active ? (active[m] ? 1 : 0) : all1;
    if (a != ctx->h_active[m]) {
      ctx->h_active[m] = a;
      changed = true;
    }
  }
  if (changed && ctx->graph_capacity > 0) {
    ctx->err = "graph mode: change the active set with cqg_set_active outside the captured call";
    return CQG_ERR_STATE;
  }
  if (changed)
    CUCHK(cudaMemcpyAsync(ctx->d_active.p, ctx->h_active.data(), ctx->nmol, cudaMemcpyHostToDevice, st));
  const double *Xg[CQG_MAXG];
  double *AXg[CQG_MAXG];
  double sJ[CQG_MAXG], sK[CQG_MAXG];
  const double *Xu[8];
  int ng, nxu;
  cqg_status s = plan_groups(ctx, nmat, X, AX, types, scale, ng, Xg, AXg, sJ, sK, nxu, Xu);
  if (s != CQG_OK) return s;
  if (ctx->graph_capacity > 0) return contract_graph(ctx, ng, Xg, AXg, sJ, sK, nxu, Xu, ctx->max_nbf, ctx->max_nbf, st);
  return contract_device(ctx, ng, Xg, AXg, sJ, sK, nxu, Xu, ctx->max_nbf, ctx->max_nbf, st);
}

cqg_status cqg_set_graph_mode(cqg_ctx *ctx, long long capacity, int max_groups) {
  if (!ctx || capacity < 0 || max_groups < 0 || max_groups > CQG_MAXG) return CQG_ERR_BAD_ARG;
  if (ctx->nshell == 0) return CQG_ERR_STATE;
  CUCHK(cudaSetDevice(ctx->device));
  ctx->graph_capacity = capacity;
  if (capacity > 0) {
    const size_t gsize = ctx->nmol > 1 ? (size_t)ctx->packed : (size_t)ctx->nbf * ctx->nbf;
    if (ctx->d_qlist.reserve((size_t)capacity) || ctx->d_qmask.reserve((size_t)capacity) ||
        ctx->d_G.reserve((size_t)std::max(max_groups, 1) * gsize)) {
      ctx->graph_capacity = 0;
      return CQG_ERR_OOM;
    }
  }
  return CQG_OK;
}

cqg_status cqg_graph_status(cqg_ctx *ctx, long long *quartets, int *overflow, int *nonfinite, int *asymmetric) {
  if (!ctx) return CQG_ERR_BAD_ARG;
  CUCHK(cudaSetDevice(ctx->device));
  CUCHK(cudaDeviceSynchronize());
  long long hr[2 * CQG_NLIST];
  int fl[4];
  CUCHK(cudaMemcpy(fl, ctx->d_flags.p, sizeof(fl), cudaMemcpyDeviceToHost));
  CUCHK(cudaMemcpy(hr, ctx->d_range.p, sizeof(hr), cudaMemcpyDeviceToHost));
  if (quartets) *quartets = hr[2 * CQG_NLIST - 1];
  if (overflow) *overflow = fl[2];
  if (nonfinite) *nonfinite = fl[0];
  if (asymmetric) *asymmetric = fl[1];
  return CQG_OK;
}

cqg_status cqg_set_active(cqg_ctx *ctx, const unsigned char *active) {
  if (!ctx) return CQG_ERR_BAD_ARG;
  if (ctx->nshell == 0) return CQG_ERR_STATE;
  CUCHK(cudaSetDevice(ctx->device));
  for (int m = 0; m < ctx->nmol; ++m) ctx->h_active[m] = active ? (active[m] ? 1 : 0) : 1;
  CUCHK(cudaMemcpy(ctx->d_active.p, ctx->h_active.data(), ctx->nmol, cudaMemcpyHostToDevice));
  return CQG_OK;
}

cqg_status cqg_autotune_next(cqg_ctx *ctx) {
  if (!ctx) return CQG_ERR_BAD_ARG;
  ctx->autotune_pending = 1;
  return CQG_OK;
}

cqg_status cqg_get_launch_shapes(cqg_ctx *ctx, int *cta_per_sm, int *warps_per_cta) {
  return cqg_get_schedule(ctx, cta_per_sm, warps_per_cta, nullptr, nullptr);
}

cqg_status cqg_get_schedule(cqg_ctx *ctx, int *cta_per_sm, int *warps_per_cta, int *quartets_per_warp,
                            int *warp_form) {
  if (!ctx) return CQG_ERR_BAD_ARG;
  for (int k = 0; k < CQG_NLIST; ++k) {
    int i, j;
    qclass_split(k % CQG_NQC, i, j);
    const bool warp = k < 2 * CQG_NQC &&
                      is_warp_class(kPairClass[i][0], kPairClass[i][1], kPairClass[j][0], kPairClass[j][1]);
    if (cta_per_sm) cta_per_sm[k] = ctx->shape_cta[k];
    if (warps_per_cta) warps_per_cta[k] = ctx->shape_wpb[k];
    if (quartets_per_warp) quartets_per_warp[k] = ctx->shape_qpw[k];
    if (warp_form) warp_form[k] = warp ? 1 : ctx->shape_var[k];
  }
  return CQG_OK;
}

cqg_status cqg_set_fusion(cqg_ctx *ctx, int tier) {
  if (!ctx) return CQG_ERR_BAD_ARG;
  if (tier < 0 || tier > 2) {
    ctx->err = "cqg_set_fusion: tier is 0 (per-class launches), 1 or 2";
    return CQG_ERR_BAD_ARG;
  }
  ctx->fused_tier = tier;
  return CQG_OK;
}

cqg_status cqg_set_siblings(cqg_ctx *ctx, int on) {
  if (!ctx) return CQG_ERR_BAD_ARG;
  ctx->siblings = on ? 1 : 0;
  select_block_table(ctx);
  return CQG_OK;
}

cqg_status cqg_set_sibling_min(cqg_ctx *ctx, int k, int min_members) {
  if (!ctx) return CQG_ERR_BAD_ARG;
  if (!class_grouped(k) || min_members < 0 || min_members == 1 || min_members > 16) {
    ctx->err = "cqg_set_sibling_min: k is a sibling class and min_members is 0 (pair tasks) or 2..16";
    return CQG_ERR_BAD_ARG;
  }
  ctx->sibling_min[k] = min_members;
  if (ctx->nshell > 0) {   // rebuild the group-mode table: the class's tasks change
    cqg_status st = build_block_tables(ctx);
    if (st != CQG_OK) return st;
  }
  return CQG_OK;
}

cqg_status cqg_get_siblings(cqg_ctx *ctx, int *on) {
  if (!ctx || !on) return CQG_ERR_BAD_ARG;
  *on = ctx->siblings;
  return CQG_OK;
}

cqg_status cqg_get_fusion(cqg_ctx *ctx, int *tier, double *tuned_ms) {
  if (!ctx) return CQG_ERR_BAD_ARG;
  if (tier) *tier = ctx->fused_tier;
  if (tuned_ms)
    for (int t = 0; t < 3; ++t) tuned_ms[t] = ctx->fusion_ms[t];
  return CQG_OK;
}

cqg_status cqg_set_schedule(cqg_ctx *ctx, const int *cta_per_sm, const int *warps_per_cta,
                            const int *quartets_per_warp, const int *warp_form) {
  if (!ctx) return CQG_ERR_BAD_ARG;
  for (int k = 0; k < CQG_NLIST; ++k) {
    if ((cta_per_sm && (cta_per_sm[k] < 0 || cta_per_sm[k] > 64)) ||
        (warps_per_cta && (warps_per_cta[k] < 0 || warps_per_cta[k] > 4)) ||
        (quartets_per_warp && (quartets_per_warp[k] < 0 || quartets_per_warp[k] > 1024)) ||
        (warp_form && warp_form[k] != 0 && warp_form[k] != 1)) {
      ctx->err = "cqg_set_schedule: entry out of range (CTAs per SM <= 64, warps per CTA <= 4, "
                 "quartets per warp <= 1024, kernel form 0 or 1)";
      return CQG_ERR_BAD_ARG;
    }
  }
  for (int k = 0; k < CQG_NLIST; ++k) {
    int i, j;
    qclass_split(k % CQG_NQC, i, j);
    const bool both = k < 2 * CQG_NQC &&
                      is_variant_class(kPairClass[i][0], kPairClass[i][1], kPairClass[j][0], kPairClass[j][1]);
    if (cta_per_sm) ctx->shape_cta[k] = cta_per_sm[k];
    if (warps_per_cta) ctx->shape_wpb[k] = warps_per_cta[k];
    if (quartets_per_warp) ctx->shape_qpw[k] = quartets_per_warp[k];
    if (warp_form && both) ctx->shape_var[k] = warp_form[k];
  }
  return CQG_OK;
}

cqg_status cqg_get_stats(cqg_ctx *ctx, cqg_stats *out) {
  if (!ctx || !out) return CQG_ERR_BAD_ARG;
  CUCHK(cudaSetDevice(ctx->device));
  CUCHK(cudaDeviceSynchronize());
  cqg_stats &s = ctx->stats;
  if (ctx->timing) {
    float ms;
    cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
    s.ms_screen = ms;
    double eri = s.ms_fused;
    for (int k = 0; k < CQG_NQC; ++k) eri += s.class_ms[k];
    s.ms_eri = eri;
    cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[3]);
    s.ms_total = ms;

  }
  *out = s;
  return CQG_OK;
}

cqg_status cqg_probe_fma_peak(int device, int fp64, double ms_target, double *tflops) {
  if (!tflops) return CQG_ERR_BAD_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return CQG_ERR_CUDA;
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  void *buf = nullptr;
  if (cudaMalloc(&buf, 64) != cudaSuccess) return CQG_ERR_OOM;
  int blocks = nsm * 8, threads = 256, iters = 256;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  float ms = 0;
  for (int rep = 0; rep < 8; ++rep) {
    cudaEventRecord(a);
    if (fp64) k_fma_probe<double><<<blocks, threads>>>((double *)buf, iters, 1.0);
    else k_fma_probe<float><<<blocks, threads>>>((float *)buf, iters, 1.0f);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    cudaEventElapsedTime(&ms, a, b);
    if (ms < ms_target && rep < 7) iters = (int)std::min(1 << 24, (int)(iters * std::max(1.5, ms_target / std::max(ms, 0.01f))));
    else break;
  }
  double flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
  *tflops = flops / (ms * 1e-3) / 1e12;
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(buf);
  return cudaGetLastError() == cudaSuccess ? CQG_OK : CQG_ERR_CUDA;
}

}  // extern "C"

// ---- One-electron integrals that allocate nothing ---------------------------------------
// The point-charge table lives in a fixed module-scope device array instead of the
// context's growable buffer.  Its device address is resolved on the first such call of a
// context, with the context's device current, and kept in the context: a context never
// outlives its device's CUDA context (a cudaDeviceReset frees every buffer a context holds,
// so it is destroyed and created again), which keeps the address from going stale.
namespace {
// Z[0..n) followed by R[n..4n) (x, y, z per charge), as k_one_e reads it
__device__ __align__(256) double g_oe_charge_table[4 * CQG_ONE_E_NOALLOC_MAX_CHARGES];

// With ctx->device current: the device address of g_oe_charge_table on that device.
cqg_status oe_charge_table(cqg_ctx *ctx, double **out) {
  if (!ctx->oe_table) {
    void *p = nullptr;
    CUCHK(cudaGetSymbolAddress(&p, g_oe_charge_table));
    ctx->oe_table = (double *)p;
  }
  *out = ctx->oe_table;
  return CQG_OK;
}
}  // namespace

extern "C" {

cqg_status cqg_one_e_noalloc(cqg_ctx *ctx, int ncharge, const double *Z, const double *R, double *S, double *T,
                             double *V, int ld, void *stream) {
  if (!ctx || ncharge < 0 || (ncharge > 0 && (!Z || !R)) || !S || !T || !V) return CQG_ERR_BAD_ARG;
  if (ncharge > CQG_ONE_E_NOALLOC_MAX_CHARGES) {
    ctx->err = "cqg_one_e_noalloc: ncharge exceeds CQG_ONE_E_NOALLOC_MAX_CHARGES (4096)";
    return CQG_ERR_BAD_ARG;
  }
  if (ctx->nshell == 0) {
    ctx->err = "cqg_set_basis has not been called";
    return CQG_ERR_STATE;
  }
  if (ctx->nmol != 1) {
    ctx->err = "cqg_one_e_noalloc is for single-molecule contexts";
    return CQG_ERR_STATE;
  }
  if (ld < ctx->nbf) {
    ctx->err = "leading dimension below the number of basis functions";
    return CQG_ERR_BAD_ARG;
  }
  CUCHK(cudaSetDevice(ctx->device));
  double *tab = nullptr;
  const cqg_status s = oe_charge_table(ctx, &tab);
  if (s != CQG_OK) return s;
  cudaStream_t st = (cudaStream_t)stream;
  // Z and R may be host or device pointers; the table is written in full for the
  // `ncharge` entries the kernel reads, so nothing in it has to start at zero.
  if (ncharge > 0) {
    CUCHK(cudaMemcpyAsync(tab, Z, (size_t)ncharge * sizeof(double), cudaMemcpyDefault, st));
    CUCHK(cudaMemcpyAsync(tab + ncharge, R, 3 * (size_t)ncharge * sizeof(double), cudaMemcpyDefault, st));
  }
  OneEShells sh;
  sh.L = ctx->d_shL.p;
  sh.nprim = ctx->d_shnp.p;
  sh.poff = ctx->d_shpoff.p;
  sh.bf = ctx->d_bf.p;
  sh.alpha = ctx->d_alpha.p;
  sh.coef = ctx->d_coef.p;
  sh.center = ctx->d_center.p;
  OneEMols om;
  memset(&om, 0, sizeof(om));
  const long long np = ctx->nallpairs;
  k_one_e<<<(unsigned)((np + 63) / 64), 64, 0, st>>>(sh, ctx->d_allpairs.p, np, ncharge, tab,
                                                     (const double3 *)(tab + ncharge), ctx->d_boys.p, S, T, V, ld,
                                                     om);
  CUCHK(cudaGetLastError());
  return CQG_OK;
}

}  // extern "C"
