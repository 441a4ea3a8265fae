// dustb_seed.cu -- seeded synthetic particles and gas on the device, with the formulas of
// athenak_b200/inputs.py (random placement): tag-keyed SplitMix64 hash draws for the
// positions (src/pgen/dust_amr/dust_setup.hpp:36-50, :114-118), species in blocks of
// ncell*ppc_s particles, Box-Muller velocity noise, uniform gas noise per cell.
#include <cstdint>

#include "dustb_common.cuh"

namespace {

__device__ __forceinline__ double hash01(uint64_t key) {
  key += 0x9E3779B97F4A7C15ull;
  key = (key ^ (key >> 30)) * 0xBF58476D1CE4E5B9ull;
  key = (key ^ (key >> 27)) * 0x94D049BB133111EBull;
  key ^= key >> 31;
  return (double)(key >> 11) * (1.0 / 9007199254740992.0);
}

constexpr uint64_t KX = 0x632BE59BD9B4E019ull, KY = 0x8CB92BAA3F3D8DD7ull;
constexpr uint64_t KZ = 0x58F38DED6F7C55B5ull, KG = 0x1D8E4E27C47D124Full;
// the stopping-time draw of the continuous distribution (dust_setup.cpp:736-745)
constexpr uint64_t KT = 0xD6E8FEB86659FD93ull;

struct SeedArgs {
  dustb_seed_desc d;
  long long start[9];     // first particle of each species
};

__global__ void k_seed_particles(double *pr, int *pi, long long stride, int npart,
                                 const double *mb, int nmb, SeedArgs a, double x1min,
                                 double x1max, double x2min, double x2max, double x3min,
                                 double x3max, int three_d) {
  long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= npart) return;
  int s = 0;
  while (s + 1 < a.d.nspecies && p >= a.start[s + 1]) ++s;
  const uint64_t tag = (uint64_t)p;
  const uint64_t key = tag + a.d.seed * 0x9E3779B97F4A7C15ull;
  const double Lx = x1max - x1min, Ly = x2max - x2min, Lz = x3max - x3min;
  double x = x1min + hash01(key + KX) * Lx;
  double y = x2min + hash01(key + KY) * Ly;
  double z = three_d ? x3min + hash01(key + KZ) * Lz : 0.5 * (x3min + x3max);
  if (three_d && a.d.hp > 0.0) {
    // Gaussian height of scale hp (Box-Muller on two draws), redrawn while outside the mesh
    for (int r = 0; r < 64; ++r) {
      const double u1 = fmax(hash01(key + KZ + 0x3333ull * (r + 1)), 1e-300);
      const double u2 = hash01(key + KZ + 0x4444ull * (r + 1));
      const double zz = a.d.hp * sqrt(-2.0 * log(u1)) * cos(2.0 * 3.141592653589793 * u2);
      if (zz >= x3min && zz < x3max) { z = zz; break; }
    }
  }
  // block by position, then the block's own half-open box decides
  int b1 = (int)((x - x1min) / Lx * a.d.nb1), b2 = (int)((y - x2min) / Ly * a.d.nb2);
  int b3 = three_d ? (int)((z - x3min) / Lz * a.d.nb3) : 0;
  b1 = min(max(b1, 0), a.d.nb1 - 1); b2 = min(max(b2, 0), a.d.nb2 - 1);
  b3 = min(max(b3, 0), a.d.nb3 - 1);
  int m = (b3 * a.d.nb2 + b2) * a.d.nb1 + b1;
  const double *sz = mb + (long long)m * 9;
  if (x < sz[0]) m -= 1; else if (x >= sz[3]) m += 1;
  sz = mb + (long long)m * 9;
  if (y < sz[1]) m -= a.d.nb1; else if (y >= sz[4]) m += a.d.nb1;
  if (three_d) {
    sz = mb + (long long)m * 9;
    if (z < sz[2]) m -= a.d.nb1 * a.d.nb2; else if (z >= sz[5]) m += a.d.nb1 * a.d.nb2;
  }
  m = min(max(m, 0), nmb - 1);
  double ts = a.d.taus[s], mass = a.d.mass[s];
  if (a.d.ts_lo > 0.0) {
    // bin s of nspecies equal bins in ln t_s; log-uniform inside it; mass ~ t_s^slope
    const double lo = log(a.d.ts_lo), w = (log(a.d.ts_hi) - lo) / a.d.nspecies;
    ts = exp(lo + ((double)s + hash01(key + KT)) * w);
    mass = a.d.mass[s] * pow(ts / exp(lo + ((double)s + 0.5) * w), a.d.mass_slope);
  }
  double v[3] = {a.d.vx[s], a.d.vy[s], a.d.vz[s]};
  if (a.d.nsh) {
    // the NSH drift of this particle's own stopping time (dust_setup.hpp:58-65)
    const double T = a.d.omega0 * ts, b = 2.0 - a.d.qshear;
    const double vx = (a.d.ug[0] + 2.0 * T * a.d.ug[1]) / (1.0 + 2.0 * b * T * T);
    const double vp = a.d.ug[1] - b * T * vx;
    v[0] = vx; v[1] = three_d ? vp : 0.0; v[2] = three_d ? 0.0 : vp;
  }
  if (a.d.vel_noise > 0.0) {
    for (int c = 0; c < 3; ++c) {
      double u1 = fmax(hash01(key + 0x1111ull * (c + 1) + KG), 1e-300);
      double u2 = hash01(key + 0x2222ull * (c + 1) + KG);
      v[c] += a.d.vel_noise * sqrt(-2.0 * log(u1)) * cos(2.0 * 3.141592653589793 * u2);
    }
  }
  auto R = [&](int r) -> double & { return pr[(long long)r * stride + p]; };
  R(DUSTB_IPX) = x; R(DUSTB_IPY) = y; R(DUSTB_IPZ) = z;
  R(DUSTB_IPVX) = v[0]; R(DUSTB_IPVY) = v[1]; R(DUSTB_IPVZ) = v[2];
  R(DUSTB_IPX1) = x; R(DUSTB_IPY1) = y; R(DUSTB_IPZ1) = z;
  R(DUSTB_IPVX1) = v[0]; R(DUSTB_IPVY1) = v[1]; R(DUSTB_IPVZ1) = v[2];
  R(DUSTB_IPRX) = 0.0; R(DUSTB_IPRY) = 0.0; R(DUSTB_IPRZ) = 0.0;
  R(DUSTB_IPTS) = ts;
  R(DUSTB_IPM) = mass;
  pi[(long long)DUSTB_PGID * stride + p] = m;
  pi[(long long)DUSTB_PTAG * stride + p] = (int)(uint32_t)(tag & 0xFFFFFFFFull);
  pi[(long long)DUSTB_PSP * stride + p] = s;
  pi[(long long)DUSTB_PLEV * stride + p] = 0;
  pi[(long long)DUSTB_PTAGH * stride + p] = (int)(uint32_t)(tag >> 32);
}

__global__ void k_seed_gas(double *u0, int nv, long long per_var, long long total, double rho0,
                           double ux, double uy, double uz, double noise, uint64_t seedkey) {
  long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;   // over nmb*per_var
  if (idx >= total) return;
  long long m = idx / per_var, c = idx - m * per_var;
  const double ug[3] = {ux, uy, uz};
  u0[(m * nv + 0) * per_var + c] = rho0;
  for (int a = 0; a < 3; ++a) {
    double val = rho0 * ug[a];
    if (noise > 0.0) {
      uint64_t k = (uint64_t)idx * 3ull + (uint64_t)a + seedkey + KG;
      val += rho0 * noise * (2.0 * hash01(k) - 1.0);
    }
    u0[(m * nv + 1 + a) * per_var + c] = val;
  }
}

}  // namespace

extern "C" int dustb_seed_uniform(const dustb_ctx *c, const dustb_seed_desc *desc, void *stream) {
  if (!c || !desc || desc->nspecies < 1 || desc->nspecies > 8) return DUSTB_EINVAL;
  const dustb_mesh &ms = c->mesh;
  if (desc->nb1 * desc->nb2 * desc->nb3 != ms.nmb) return DUSTB_EINVAL;
  dustb::Ind d = dustb::make_ind(ms);
  const long long ncell = (long long)ms.nmb * d.nx1 * d.nx2 * d.nx3;
  SeedArgs a;
  a.d = *desc;
  long long tot = 0;
  for (int s = 0; s < desc->nspecies; ++s) { a.start[s] = tot; tot += ncell * desc->ppc[s]; }
  for (int s = desc->nspecies; s < 9; ++s) a.start[s] = tot;
  if (tot != c->part.npart || tot > c->part.stride) return DUSTB_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  if (tot > 0) {
    unsigned nb = (unsigned)((tot + 255) / 256);
    k_seed_particles<<<nb, 256, 0, st>>>(c->part.pr, c->part.pi, c->part.stride, (int)tot,
                                         ms.mb_size, ms.nmb, a, ms.x1min, ms.x1max, ms.x2min,
                                         ms.x2max, ms.x3min, ms.x3max, ms.three_d);
  }
  const long long per_var = d.cells();
  const long long total = per_var * ms.nmb;
  const uint64_t seedkey = desc->seed * 0x9E3779B97F4A7C15ull;
  k_seed_gas<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(
      c->f.u0, c->f.nvar_gas, per_var, total, desc->rho0, desc->ug[0], desc->ug[1], desc->ug[2],
      desc->gas_noise, seedkey);
  return dustb_host::launch_status("seed_uniform");
}
