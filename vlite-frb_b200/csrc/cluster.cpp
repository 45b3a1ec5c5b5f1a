// Friends-of-friends clustering of candidates across DM trials and time (a
// new-build extension: the reference stops at calcstats' per-DM peak flag).
//
// Two candidates are friends when their trial indices differ by at most
// dm_tol and their sample intervals [t, t + width) are at most t_tol samples
// apart: max(t_a, t_b) - min(t_a + w_a, t_b + w_b) <= t_tol (overlapping
// intervals have a negative gap).  Clusters are the connected components of that
// relation; each is reported by its brightest member (ties: the lower trial
// index, then the earlier t), and the clusters are listed by that member's
// t, then trial index.  The candidates a chunk-by-chunk search emits for one
// pulse -- neighbouring trials, neighbouring chunks -- collapse to one.
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <numeric>
#include <vector>

#include "../../include/vfrb.h"

namespace {

struct Dsu {
  std::vector<int32_t> p;
  explicit Dsu(int32_t n) : p((size_t)n) { std::iota(p.begin(), p.end(), 0); }
  int32_t find(int32_t a) {
    while (p[(size_t)a] != a) {
      p[(size_t)a] = p[(size_t)p[(size_t)a]];
      a = p[(size_t)a];
    }
    return a;
  }
  void join(int32_t a, int32_t b) {
    a = find(a);
    b = find(b);
    if (a != b) p[(size_t)std::max(a, b)] = std::min(a, b);
  }
};

// a outranks b as a cluster's representative
bool brighter(const vfrb_cand& a, const vfrb_cand& b) {
  if (a.snr != b.snr) return a.snr > b.snr;
  if (a.dm_index != b.dm_index) return a.dm_index < b.dm_index;
  return a.t < b.t;
}

}  // namespace

extern "C" int vfrb_cluster_cands(const vfrb_cand* in, int32_t n, int32_t dm_tol, int64_t t_tol, vfrb_cand* out,
                                  int32_t* nout, int32_t* cluster_of) {
  if (!nout || n < 0 || (n > 0 && (!in || !out)) || dm_tol < 0 || t_tol < 0) return VFRB_ERR_ARG;
  *nout = 0;
  for (int32_t i = 0; i < n; ++i)
    if (in[i].width < 1 || !(in[i].snr == in[i].snr)) return VFRB_ERR_ARG;
  if (n == 0) return VFRB_OK;
  // sweep in start order; `open` holds the candidates whose interval end plus
  // t_tol still reaches the current start
  std::vector<int32_t> order((size_t)n);
  std::iota(order.begin(), order.end(), 0);
  std::sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
    return in[a].t != in[b].t ? in[a].t < in[b].t : a < b;
  });
  Dsu dsu(n);
  std::vector<int32_t> open;
  for (const int32_t i : order) {
    const vfrb_cand& c = in[i];
    size_t k = 0;
    for (const int32_t j : open) {
      const vfrb_cand& o = in[j];
      if (o.t + o.width + t_tol < c.t) continue;  // closed for this and every later start
      open[k++] = j;
      if (std::abs((int64_t)o.dm_index - c.dm_index) <= dm_tol) dsu.join(i, j);
    }
    open.resize(k);
    open.push_back(i);
  }
  // representative per component
  std::vector<int32_t> best((size_t)n, -1);
  for (int32_t i = 0; i < n; ++i) {
    const int32_t r = dsu.find(i);
    if (best[(size_t)r] < 0 || brighter(in[i], in[best[(size_t)r]])) best[(size_t)r] = i;
  }
  std::vector<int32_t> reps;
  for (int32_t i = 0; i < n; ++i)
    if (dsu.find(i) == i) reps.push_back(i);
  std::sort(reps.begin(), reps.end(), [&](int32_t a, int32_t b) {
    const vfrb_cand& x = in[best[(size_t)a]];
    const vfrb_cand& y = in[best[(size_t)b]];
    return x.t != y.t ? x.t < y.t : x.dm_index < y.dm_index;
  });
  std::vector<int32_t> label((size_t)n, -1);
  std::vector<vfrb_cand> res(reps.size());  // out may alias in
  for (size_t k = 0; k < reps.size(); ++k) {
    label[(size_t)reps[k]] = (int32_t)k;
    res[k] = in[best[(size_t)reps[k]]];
  }
  if (cluster_of)
    for (int32_t i = 0; i < n; ++i) cluster_of[i] = label[(size_t)dsu.find(i)];
  std::copy(res.begin(), res.end(), out);
  *nout = (int32_t)reps.size();
  return VFRB_OK;
}
