// Host shim over chronusq_public_b200/csrc/siblings.h for the CPU tests: the shell families
// and the sibling groups of one pair list, through a C ABI.
#include "siblings.h"

extern "C" {

int sib_families(int nshell, const int *L, const int *nprim, const int *poff, const double *alpha,
                 const double *centers, const int *mol, int *fam) {
  const std::vector<int> f = cqg_sib::shell_families(nshell, L, nprim, poff, alpha, centers, mol);
  int nf = 0;
  for (int s = 0; s < nshell; ++s) {
    fam[s] = f[s];
    nf = f[s] + 1 > nf ? f[s] + 1 : nf;
  }
  return nf;
}

int sib_pair_groups(int n, const int *a, const int *b, const int *L, int nshell, const int *fam, int cap, int *gid,
                    int *rank) {
  std::vector<int> f(fam, fam + nshell), g, r;
  const int ng = cqg_sib::pair_groups(n, a, b, L, f, cap, g, r);
  for (int k = 0; k < n; ++k) {
    gid[k] = g[k];
    rank[k] = r[k];
  }
  return ng;
}

}  // extern "C"
