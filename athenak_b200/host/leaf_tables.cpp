// leaf_tables.cpp -- host build of the leaf traversal's block geometry (see leaf_tables.hpp).
// Reference: DustGasDrag::BuildLeafTraversal3D, src/dust/dust_cloud3d.cpp:604-650 (finest-cell
// boxes and levels), :651-731 (the distinct neighbours from the 56 slots and their periodic
// shifts), :732-776 (nbmax and the ring the neighbours hold), :777-793 (the location index).
#include "leaf_tables.hpp"

#include <algorithm>
#include <utility>

namespace dustb_host {
namespace {

// NeighborIndex (src/mesh/nghbr_index.hpp:29-60) of direction (ix, iy, iz), sub-slots n1, n2
int slot_of(int ix, int iy, int iz, int n1, int n2) {
  const int ax = ix < 0 ? -ix : ix, ay = iy < 0 ? -iy : iy;
  if (iz == 0) {
    if (ix * iy == 0) return ax * 2 * (ix + 1) + ay * 2 * (iy + 5) + n1 + 2 * n2;
    return 16 + (ix + 1) + 2 * (iy + 1) + n1;
  }
  if (ix * iy == 0) return 24 + ax * (ix + 9) + ay * (iy + 17) + 2 * (iz + 1) + n1 + 2 * n2;
  return 48 + (ix + 1) / 2 + (iy + 1) + 2 * (iz + 1);
}

// the crossing direction of each of the 56 slots
void slot_dirs(int dir[56][3]) {
  for (int n = 0; n < 56; ++n) dir[n][0] = dir[n][1] = dir[n][2] = 0;
  for (int iz = -1; iz <= 1; ++iz)
    for (int iy = -1; iy <= 1; ++iy)
      for (int ix = -1; ix <= 1; ++ix) {
        const int nd = (ix != 0) + (iy != 0) + (iz != 0);
        if (nd == 0) continue;
        // faces: two sub-slot indices; edges: one; corners: none
        for (int n2 = 0; n2 <= (nd == 1 ? 1 : 0); ++n2)
          for (int n1 = 0; n1 <= (nd <= 2 ? 1 : 0); ++n1) {
            const int s = slot_of(ix, iy, iz, n1, n2);
            dir[s][0] = ix; dir[s][1] = iy; dir[s][2] = iz;
          }
      }
}

// num / den rounded half away from zero (den > 0), as lround of the quotient
long long round_div(long long num, long long den) {
  return num >= 0 ? (2 * num + den) / (2 * den) : -((-2 * num + den) / (2 * den));
}

}  // namespace

bool BuildLeafTables(const LeafGeometry &g, int nmb, const int *lloc, const int *nghbr56,
                     LeafTablesHost &out) {
  out = LeafTablesHost();
  if (nmb <= 0 || !lloc || !nghbr56 || g.max_level < g.root_level) return false;
  for (int d = 0; d < 3; ++d)
    if (g.nx[d] < 1 || g.nmbroot[d] < 1) return false;
  const int nlev = g.max_level - g.root_level;
  if (nlev > 16) return false;
  out.nlev = nlev;
  for (int d = 0; d < 3; ++d) out.nfine[d] = (g.nmbroot[d] * g.nx[d]) << nlev;
  out.fbox.assign((size_t)nmb * 6, 0);
  out.blev.assign(nmb, 0);
  for (int b = 0; b < nmb; ++b) {
    const int dl = lloc[4 * b] - g.root_level;
    if (dl < 0 || dl > nlev) return false;
    out.blev[b] = dl;
    const int ratio = 1 << (nlev - dl);
    for (int d = 0; d < 3; ++d) {
      const int lx = lloc[4 * b + 1 + d];
      if (lx < 0 || lx >= (g.nmbroot[d] << dl)) return false;
      out.fbox[6 * b + 2 * d] = lx * g.nx[d] * ratio;
      out.fbox[6 * b + 2 * d + 1] = out.fbox[6 * b + 2 * d] + g.nx[d] * ratio;
    }
  }
  int dir[56][3];
  slot_dirs(dir);
  out.nnb.assign(nmb, 0);
  out.nb.assign((size_t)nmb * kLeafMaxNb, -1);
  out.nbs.assign((size_t)nmb * kLeafMaxNb * 3, 0);
  for (int m = 0; m < nmb; ++m) {
    const int *fm = &out.fbox[6 * m];
    int c = 0;
    for (int n = 0; n < 56; ++n) {
      const int b = nghbr56[56 * m + n];
      if (b < 0) continue;
      if (b >= nmb) return false;
      const int *fb = &out.fbox[6 * b];
      int s[3];
      for (int d = 0; d < 3; ++d) {
        // across the slot's direction the gap between the facing sides (0 or a domain length);
        // along it the image whose centre is nearest
        const int id = dir[n][d];
        const long long N = out.nfine[d];
        if (id > 0) s[d] = (int)round_div((long long)fb[2 * d] - fm[2 * d + 1], N);
        else if (id < 0) s[d] = (int)round_div((long long)fb[2 * d + 1] - fm[2 * d], N);
        else
          s[d] = (int)round_div((long long)fb[2 * d] + fb[2 * d + 1] - fm[2 * d] - fm[2 * d + 1],
                                2 * N);
      }
      bool seen = (b == m && s[0] == 0 && s[1] == 0 && s[2] == 0);
      for (int k = 0; k < c && !seen; ++k) {
        const int *q = &out.nbs[((size_t)m * kLeafMaxNb + k) * 3];
        seen = out.nb[(size_t)m * kLeafMaxNb + k] == b && q[0] == s[0] && q[1] == s[1] &&
               q[2] == s[2];
      }
      if (seen) continue;
      if (c >= kLeafMaxNb) return false;
      out.nb[(size_t)m * kLeafMaxNb + c] = b;
      for (int d = 0; d < 3; ++d) out.nbs[((size_t)m * kLeafMaxNb + c) * 3 + d] = s[d];
      ++c;
    }
    out.nnb[m] = c;
  }
  out.nbmax.assign(nmb, 0);
  out.safe.assign((size_t)nmb * 3, 0);
  for (int m = 0; m < nmb; ++m) {
    const int nn = out.nnb[m];
    const int *nbm = &out.nb[(size_t)m * kLeafMaxNb];
    const int *sm = &out.nbs[(size_t)m * kLeafMaxNb * 3];
    int mx = out.blev[m];
    int w[3] = {0, 0, 0};
    for (int k = 0; k < nn; ++k) {
      const int *fb = &out.fbox[6 * nbm[k]];
      mx = std::max(mx, out.blev[nbm[k]]);
      for (int d = 0; d < 3; ++d) {
        const int wd = fb[2 * d + 1] - fb[2 * d];
        w[d] = (k == 0 || wd < w[d]) ? wd : w[d];
      }
    }
    out.nbmax[m] = mx;
    // every cell of the ring of width w around the block must lie inside one neighbour image
    const int *fm = &out.fbox[6 * m];
    bool ok = w[0] > 0 && w[1] > 0 && w[2] > 0;
    for (int d = 0; d < 3 && ok; ++d) ok = (fm[2 * d + 1] - fm[2 * d]) % w[d] == 0;
    for (int cz = fm[4] - w[2]; ok && cz < fm[5] + w[2]; cz += w[2])
      for (int cy = fm[2] - w[1]; ok && cy < fm[3] + w[1]; cy += w[1])
        for (int cx = fm[0] - w[0]; ok && cx < fm[1] + w[0]; cx += w[0]) {
          if (cx >= fm[0] && cx < fm[1] && cy >= fm[2] && cy < fm[3] && cz >= fm[4] &&
              cz < fm[5])
            continue;
          if (!g.x3per && (cz < 0 || cz >= out.nfine[2])) continue;
          bool held = false;
          for (int k = 0; k < nn && !held; ++k) {
            const int *fb = &out.fbox[6 * nbm[k]];
            const int *s = &sm[3 * k];
            const int lo[3] = {fb[0] - s[0] * out.nfine[0], fb[2] - s[1] * out.nfine[1],
                               fb[4] - s[2] * out.nfine[2]};
            const int hi[3] = {fb[1] - s[0] * out.nfine[0], fb[3] - s[1] * out.nfine[1],
                               fb[5] - s[2] * out.nfine[2]};
            held = lo[0] <= cx && cx + w[0] <= hi[0] && lo[1] <= cy && cy + w[1] <= hi[1] &&
                   lo[2] <= cz && cz + w[2] <= hi[2];
          }
          ok = held;
        }
    if (!ok) { w[0] = w[1] = w[2] = 0; ++out.nunsafe; }
    for (int d = 0; d < 3; ++d) out.safe[3 * m + d] = w[d];
  }
  std::vector<std::pair<std::int64_t, int>> kv(nmb);
  for (int b = 0; b < nmb; ++b) {
    const int sh = nlev - out.blev[b];
    const int *fb = &out.fbox[6 * b];
    kv[b] = {LeafLocKey(out.blev[b], fb[0] / (g.nx[0] << sh), fb[2] / (g.nx[1] << sh),
                        fb[4] / (g.nx[2] << sh)), b};
  }
  std::sort(kv.begin(), kv.end());
  out.lockey.resize(nmb);
  out.locblk.resize(nmb);
  for (int k = 0; k < nmb; ++k) { out.lockey[k] = kv[k].first; out.locblk[k] = kv[k].second; }
  return true;
}

}  // namespace dustb_host

extern "C" int dustb_host_leaf_tables(const int *geo, int nmb, const int *lloc,
                                      const int *nghbr56, int *info, int *fbox, int *blev,
                                      int *nnb, int *nb, int *nbs, int *nbmax, int *safe,
                                      long long *lockey, int *locblk) {
  if (!geo || !info || !fbox || !blev || !nnb || !nb || !nbs || !nbmax || !safe || !lockey ||
      !locblk)
    return -1;
  dustb_host::LeafGeometry g;
  for (int d = 0; d < 3; ++d) { g.nx[d] = geo[d]; g.nmbroot[d] = geo[3 + d]; }
  g.root_level = geo[6]; g.max_level = geo[7]; g.x3per = geo[8];
  dustb_host::LeafTablesHost h;
  if (!dustb_host::BuildLeafTables(g, nmb, lloc, nghbr56, h)) return -1;
  info[0] = h.nlev;
  for (int d = 0; d < 3; ++d) info[1 + d] = h.nfine[d];
  info[4] = h.nunsafe;
  std::copy(h.fbox.begin(), h.fbox.end(), fbox);
  std::copy(h.blev.begin(), h.blev.end(), blev);
  std::copy(h.nnb.begin(), h.nnb.end(), nnb);
  std::copy(h.nb.begin(), h.nb.end(), nb);
  std::copy(h.nbs.begin(), h.nbs.end(), nbs);
  std::copy(h.nbmax.begin(), h.nbmax.end(), nbmax);
  std::copy(h.safe.begin(), h.safe.end(), safe);
  for (int k = 0; k < nmb; ++k) lockey[k] = (long long)h.lockey[k];
  std::copy(h.locblk.begin(), h.locblk.end(), locblk);
  return 0;
}
