// dep_plan.cpp -- host build of the general deposit remap (see dep_plan.hpp).
// Reference: DepRemapPlan's static part, src/bvals/bvals_dep_general.cpp:62-160 (block boxes in
// finest units, the per-direction overlaps with the periodic wrap and the x3 mirror),
// :163-231 (the overlaps of a block pair), :383-545 (pairs of a target with itself and its
// neighbours, the coverage check, the target lists ordered by target, source gid, source cell).
#include "dep_plan.hpp"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <tuple>

namespace dustb_host {
namespace {

using i64 = std::int64_t;

struct Box {
  int gid = 0, level = 0;
  i64 lo[3] = {0, 0, 0};   // active box in finest-level units
  i64 sc = 1;              // cell width in those units
};

// one piece of a source interval inside a target cell along one direction
struct Piece { int t; i64 len; };

// The pieces of source index q (0 .. nx + 2 ng - 1) of block s along direction d inside the
// active cells of block t.  A source interval outside the domain is moved back by one period
// (periodic), or mirrored about the face (x3 fold), or dropped (x3 drop).
void pieces(const DepPlanGeometry &g, const i64 N[3], const Box &s, const Box &t, int d, int q,
            std::vector<Piece> &out) {
  out.clear();
  i64 a = s.lo[d] + (i64)(q - g.ng) * s.sc, b = a + s.sc;
  if (d == 2 && g.x3mode != 0 && (a < 0 || a >= N[2])) {
    if (g.x3mode == 2) return;
    const i64 lo = a, hi = b;
    if (lo < 0) { a = -hi; b = -lo; } else { a = 2 * N[2] - hi; b = 2 * N[2] - lo; }
  } else if (a < 0) {
    a += N[d]; b += N[d];
  } else if (a >= N[d]) {
    a -= N[d]; b -= N[d];
  }
  const i64 tlo = t.lo[d], thi = t.lo[d] + (i64)g.nx[d] * t.sc;
  const i64 lo = std::max(a, tlo), hi = std::min(b, thi);
  if (hi <= lo) return;
  for (i64 c = (lo - tlo) / t.sc; c <= (hi - 1 - tlo) / t.sc; ++c) {
    const i64 clo = tlo + c * t.sc;
    const i64 len = std::min(b, clo + t.sc) - std::max(a, clo);
    if (len > 0) out.push_back({(int)c, len});
  }
}

struct Ent { int tflat, sgid, scell; double w; };

}  // namespace

bool BuildDepPlan(const DepPlanGeometry &g, int nmb, const int *lloc, const int *nghbr56,
                  DepPlanHost &out) {
  out = DepPlanHost();
  if (nmb <= 0 || !lloc || !nghbr56 || g.ng < 1 || g.max_level < g.root_level) return false;
  for (int d = 0; d < 3; ++d)
    if (g.nx[d] < 2 * g.ng || g.nmbroot[d] < 1) return false;
  const int nc[3] = {g.nx[0] + 2 * g.ng, g.nx[1] + 2 * g.ng, g.nx[2] + 2 * g.ng};
  const int ncell = nc[0] * nc[1] * nc[2];
  if ((long long)nmb * ncell > 2147483647LL) return false;
  i64 N[3];
  for (int d = 0; d < 3; ++d)
    N[d] = (i64)g.nmbroot[d] * g.nx[d] * ((i64)1 << (g.max_level - g.root_level));
  std::vector<Box> box(nmb);
  for (int m = 0; m < nmb; ++m) {
    const int *l = lloc + 4 * m;
    if (l[0] < g.root_level || l[0] > g.max_level) return false;
    Box &b = box[m];
    b.gid = m; b.level = l[0];
    b.sc = (i64)1 << (g.max_level - l[0]);
    for (int d = 0; d < 3; ++d) b.lo[d] = (i64)l[1 + d] * g.nx[d] * b.sc;
  }
  std::vector<Ent> ent;
  std::vector<double> cov((size_t)nmb * ncell, 0.0);
  std::vector<Piece> p1[64], p2[64], p3[64];   // (per source index; nc <= 64 checked below)
  for (int d = 0; d < 3; ++d) if (nc[d] > 64) return false;
  for (int tm = 0; tm < nmb; ++tm) {
    const Box &t = box[tm];
    std::vector<int> cand{tm};
    for (int n = 0; n < 56; ++n) {
      const int s = nghbr56[(size_t)tm * 56 + n];
      if (s >= 0 && s < nmb) cand.push_back(s);
    }
    std::sort(cand.begin(), cand.end());
    cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
    const double tvol = (double)t.sc * (double)t.sc * (double)t.sc;
    for (const int sm : cand) {
      const Box &s = box[sm];
      for (int i = 0; i < nc[0]; ++i) pieces(g, N, s, t, 0, i, p1[i]);
      for (int j = 0; j < nc[1]; ++j) pieces(g, N, s, t, 1, j, p2[j]);
      for (int k = 0; k < nc[2]; ++k) pieces(g, N, s, t, 2, k, p3[k]);
      for (int k = 0; k < nc[2]; ++k) {
        if (p3[k].empty()) continue;
        const bool kin = k >= g.ng && k < nc[2] - g.ng;
        for (int j = 0; j < nc[1]; ++j) {
          if (p2[j].empty()) continue;
          const bool jin = j >= g.ng && j < nc[1] - g.ng;
          for (int i = 0; i < nc[0]; ++i) {
            if (p1[i].empty()) continue;
            if (kin && jin && i >= g.ng && i < nc[0] - g.ng) continue;   // an active cell
            const int scell = (k * nc[1] + j) * nc[0] + i;
            for (const Piece &z : p3[k])
              for (const Piece &y : p2[j])
                for (const Piece &x : p1[i]) {
                  const double vol = (double)x.len * (double)y.len * (double)z.len;
                  const int tcell = ((z.t + g.ng) * nc[1] + (y.t + g.ng)) * nc[0] + (x.t + g.ng);
                  ent.push_back({tm * ncell + tcell, sm, scell, vol / tvol});
                  cov[(size_t)sm * ncell + scell] += vol;
                }
          }
        }
      }
    }
  }
  // every source ghost cell covered exactly once (but those dropped beyond a physical x3 face)
  for (int sm = 0; sm < nmb; ++sm) {
    const Box &s = box[sm];
    const double svol = (double)s.sc * (double)s.sc * (double)s.sc;
    for (int k = 0; k < nc[2]; ++k)
      for (int j = 0; j < nc[1]; ++j)
        for (int i = 0; i < nc[0]; ++i) {
          const bool act = i >= g.ng && i < nc[0] - g.ng && j >= g.ng && j < nc[1] - g.ng &&
                           k >= g.ng && k < nc[2] - g.ng;
          if (act) continue;
          const i64 z0 = s.lo[2] + (i64)(k - g.ng) * s.sc;
          if (g.x3mode == 2 && (z0 < 0 || z0 >= N[2])) continue;
          const double c = cov[(size_t)sm * ncell + (k * nc[1] + j) * nc[0] + i];
          if (std::fabs(c - svol) / svol > 1e-9) ++out.nbad;
        }
  }
  std::sort(ent.begin(), ent.end(), [](const Ent &x, const Ent &y) {
    return std::tie(x.tflat, x.sgid, x.scell) < std::tie(y.tflat, y.sgid, y.scell);
  });
  out.ent_src.resize(ent.size());
  out.ent_w.resize(ent.size());
  for (size_t e = 0; e < ent.size(); ++e) {
    if (e == 0 || ent[e].tflat != ent[e - 1].tflat) {
      out.seg_tgt.push_back(ent[e].tflat);
      out.seg_ptr.push_back((int)e);
    }
    out.ent_src[e] = ent[e].sgid * ncell + ent[e].scell;
    out.ent_w[e] = ent[e].w;
  }
  out.seg_ptr.push_back((int)ent.size());
  return true;
}

}  // namespace dustb_host

extern "C" int dustb_host_dep_plan(const int *geo, int nmb, const int *lloc, const int *nghbr56,
                                   int *counts, int *seg_tgt, int *seg_ptr, int *ent_src,
                                   double *ent_w, long long cap_seg, long long cap_ent) {
  if (!geo || !counts) return -1;
  dustb_host::DepPlanGeometry g;
  for (int d = 0; d < 3; ++d) { g.nx[d] = geo[d]; g.nmbroot[d] = geo[4 + d]; }
  g.ng = geo[3]; g.root_level = geo[7]; g.max_level = geo[8]; g.x3mode = geo[9];
  if (g.x3mode < 0 || g.x3mode > 2) return -1;
  dustb_host::DepPlanHost h;
  if (!dustb_host::BuildDepPlan(g, nmb, lloc, nghbr56, h)) return -1;
  const long long nseg = (long long)h.seg_tgt.size(), nent = (long long)h.ent_src.size();
  counts[0] = (int)nseg; counts[1] = (int)nent; counts[2] = h.nbad;
  if (!seg_tgt || !seg_ptr || !ent_src || !ent_w) return 0;
  if (cap_seg < nseg || cap_ent < nent) return -3;
  std::copy(h.seg_tgt.begin(), h.seg_tgt.end(), seg_tgt);
  std::copy(h.seg_ptr.begin(), h.seg_ptr.end(), seg_ptr);
  std::copy(h.ent_src.begin(), h.ent_src.end(), ent_src);
  std::copy(h.ent_w.begin(), h.ent_w.end(), ent_w);
  return 0;
}
