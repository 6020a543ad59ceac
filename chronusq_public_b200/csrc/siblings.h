// Sibling groups of shell pairs: the host-side rules of the engine's shared-primitive
// evaluation (plain C++, no CUDA types).
//
// A segmented basis stores the functions of one general contraction as separate shells with
// the same exponents and different coefficients (cc-pVXZ: the 1s and 2s shells of a
// first-row atom).  Two shell pairs whose shells have the same centres, angular momenta and
// exponents have the same primitive integrals; only the coefficient weights differ.  The
// engine evaluates such sibling pairs from one pass over the shared primitive pairs.
#pragma once
#include <cstdint>
#include <cstring>
#include <map>
#include <utility>
#include <vector>

namespace cqg_sib {

// Family id of every shell: shells of one molecule with the same centre, angular momentum
// and primitive exponents (compared bit for bit) share a family.
inline std::vector<int> shell_families(int nshell, const int *L, const int *nprim, const int *poff,
                                       const double *alpha, const double *centers, const int *mol) {
  std::map<std::vector<uint64_t>, int> ids;
  std::vector<int> fam(nshell);
  for (int s = 0; s < nshell; ++s) {
    std::vector<uint64_t> key;
    key.push_back((uint64_t)mol[s]);
    key.push_back((uint64_t)L[s]);
    key.push_back((uint64_t)nprim[s]);
    for (int x = 0; x < 3; ++x) {
      uint64_t u;
      std::memcpy(&u, &centers[3 * s + x], sizeof(u));
      key.push_back(u);
    }
    for (int k = 0; k < nprim[s]; ++k) {
      uint64_t u;
      std::memcpy(&u, &alpha[poff[s] + k], sizeof(u));
      key.push_back(u);
    }
    fam[s] = ids.emplace(key, (int)ids.size()).first->second;
  }
  return fam;
}

// Sibling groups of the n pairs (a[k], b[k]) of one pair class (orientation L_a >= L_b):
// pairs whose shells come from the same two families (unordered when L_a == L_b), in their
// given order, cut into groups of at most `cap` members.  Returns the number of groups;
// gid[k] = group of pair k (groups numbered by their first pair), rank[k] = its member
// index.  cap = 1 leaves every pair on its own.
inline int pair_groups(int n, const int *a, const int *b, const int *L, const std::vector<int> &fam, int cap,
                       std::vector<int> &gid, std::vector<int> &rank) {
  gid.assign(n, -1);
  rank.assign(n, 0);
  std::map<std::pair<int, int>, std::pair<int, int>> open;   // family pair -> (group, members so far)
  int ng = 0;
  for (int k = 0; k < n; ++k) {
    if (cap <= 1) {
      gid[k] = ng++;
      continue;
    }
    int fa = fam[a[k]], fb = fam[b[k]];
    if (L[a[k]] == L[b[k]] && fa < fb) std::swap(fa, fb);
    auto it = open.find(std::make_pair(fa, fb));
    if (it == open.end() || it->second.second >= cap) {
      open[std::make_pair(fa, fb)] = std::make_pair(ng, 1);
      gid[k] = ng++;
    } else {
      gid[k] = it->second.first;
      rank[k] = it->second.second++;
    }
  }
  return ng;
}

// Whether member pair (ma, mb) of a group led by (la_sh, lb_sh) is stored with its shells
// in the leader's order (shell ma from the family of la_sh).  Only s-s pairs of two
// families can be swapped; their integrals are symmetric in the two shells.
inline bool same_orientation(int ma, int la_sh, const std::vector<int> &fam) { return fam[ma] == fam[la_sh]; }

}  // namespace cqg_sib
