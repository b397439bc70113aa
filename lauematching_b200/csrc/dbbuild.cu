// DB build: forward simulation of the orientation DB on the device.
//
// Restates the per-orientation loop of LaueMatchingCPU.c:595-667 (the only
// implementation in the reference, copied at LaueMatchingGPU.cu:478-614 and
// LaueMatchingGPUStream.cu:854-946).  One thread owns one orientation and
// walks the HKL list in file order, appending on-detector, in-band,
// not-yet-seen pixels until MaxNrLaueSpots are taken.
//
// Arithmetic.  Each (orientation, HKL) pair is first screened in FP32 with
// FMA.  The screen only REJECTS: a pair is dropped when, with an error
// margin far above the FP32 error of the chain, it is certainly behind the
// detector, off the detector or outside the energy band.  Every other pair
// is recomputed in FP64 with the reference's exact operation order and
// rounding (no FMA; C truncation of the pixel coordinate as x86 performs
// it), and that result alone decides acceptance and the pixel.  The records
// are therefore identical to the reference's, byte for byte; a build flag
// (exact_all) runs the FP64 path for every pair to check the screen.
//
// Layout.  Blocks of TB orientations; the HKL list is staged through shared
// memory in chunks (broadcast reads); accepted pixels live in shared memory
// as [spot][thread] so the de-duplication scan is bank-conflict free; the
// block's records (contiguous in the DB) are written with coalesced stores.
#include <climits>
#include <cmath>

#include "kernels.cuh"

namespace lmb {

struct BuildGeo {
  double recip[9], rt[9];
  double p0, p1, p2, px_x, px_y, cx, cy, elo, ehi;
  int W, H, S, R;
  float rtf[9];
  float p0f, p1f, p2f, inv_pxxf, inv_pyf, cxf, cyf, elof, ehif, hc4pif;
  float tolx, toly;  // FP32 pixel-error scale: 1e-4 * p2 / |px|
};

static constexpr double kHcKeVnm = 1.2398419739;              // LaueMatchingHeaders.h:41
static constexpr double kFourPi = 4.0 * 3.14159265358979323846;  // 4 * M_PI as C folds it
static constexpr int kHklChunk = 512;

// FP32 screen: false only when the pair is certainly rejected in FP64.
// Ordered cheapest-first: the energy band needs only q (E = c*|q|^2/(-q_z),
// c = hc/4pi, tested by multiplication), which rejects most pairs before the
// detector projection is computed.  Margins: the FP32 chain has relative
// error ~1e-6 in |q|^2 and absolute ~2e-6*|q| in q_z, ~3e-6 in the unit
// vectors; every test below leaves >= 30x that.
__device__ __forceinline__ bool screen(const float T[9], const float4 hf, const BuildGeo &g) {
  const float qx = fmaf(T[0], hf.x, fmaf(T[1], hf.y, T[2] * hf.z));
  const float qy = fmaf(T[3], hf.x, fmaf(T[4], hf.y, T[5] * hf.z));
  const float qz = fmaf(T[6], hf.x, fmaf(T[7], hf.y, T[8] * hf.z));
  const float ql2 = fmaf(qx, qx, fmaf(qy, qy, qz * qz));
  if (!(ql2 > 1e-30f) || !(ql2 < 1e30f)) return true;  // let FP64 decide
  const float rq = rsqrtf(ql2);
  const float ql = ql2 * rq;
  const float nq = -qz;   // |q| sin(theta)
  const float s = nq * rq;  // sin(theta)
  if (fabsf(s) >= 1e-5f) {
    const float cq = g.hc4pif * ql2;  // E * (-q_z)
    if (s < 0.f) {
      if (g.elof > 0.f) return false;  // E < 0 < Elo
    } else {
      if (g.ehif > 0.f && cq > g.ehif * fmaf(nq, 1e-4f, nq) + g.ehif * 1e-4f * ql) return false;
      if (g.elof > 0.f && cq < g.elof * fmaf(nq, -1e-4f, nq) - g.elof * 1e-4f * ql) return false;
    }
  }
  const float hx = qx * rq, hy = qy * rq, hz = qz * rq;
  const float td = -2.f * hz;
  const float k0 = td * hx, k1 = td * hy, k2 = fmaf(td, hz, 1.f);
  const float z = fmaf(g.rtf[6], k0, fmaf(g.rtf[7], k1, g.rtf[8] * k2));
  if (z < -1e-4f) return false;  // xyz[2] <= 0 for sure
  if (z <= 1e-4f) return true;   // too close to call
  const float iz = __fdividef(1.f, z);
  const float x = fmaf(g.rtf[0], k0, fmaf(g.rtf[1], k1, g.rtf[2] * k2)) * iz;
  const float y = fmaf(g.rtf[3], k0, fmaf(g.rtf[4], k1, g.rtf[5] * k2)) * iz;
  // pixel = (x/z * p2 - p0) / px + (N-1)/2 ; accepted iff trunc in [0, N-1],
  // i.e. pixel in (-1, N).  |error| <= 3e-6 (1+|x/z|)/z * p2/px (FP32 chain),
  // the margin below is ~30x that plus 0.05 px.
  const float pxv = fmaf(fmaf(x, g.p2f, -g.p0f), g.inv_pxxf, g.cxf);
  const float tx = fmaf(g.tolx * (1.f + fabsf(x)), iz, 0.05f);
  if (pxv < -1.f - tx || pxv > (float)g.W + tx) return false;
  const float pyv = fmaf(fmaf(y, g.p2f, -g.p1f), g.inv_pyf, g.cyf);
  const float ty = fmaf(g.toly * (1.f + fabsf(y)), iz, 0.05f);
  if (pyv < -1.f - ty || pyv > (float)g.H + ty) return false;
  return true;
}

// FP64 evaluation in the reference's exact order (LaueMatchingCPU.c:605-636,
// MatrixMultF LaueMatchingHeaders.h:361-369).  Returns acceptance and pixel.
__device__ __forceinline__ bool exact_spot(const double T[9], const int4 hk, const BuildGeo &g,
                                           int &ipx, int &ipy) {
  const double h = (double)hk.x, k = (double)hk.y, l = (double)hk.z;
  const double q0 = dadd(dadd(dadd(0.0, dmul(T[0], h)), dmul(T[1], k)), dmul(T[2], l));
  const double q1 = dadd(dadd(dadd(0.0, dmul(T[3], h)), dmul(T[4], k)), dmul(T[5], l));
  const double q2 = dadd(dadd(dadd(0.0, dmul(T[6], h)), dmul(T[7], k)), dmul(T[8], l));
  const double ql = dsqrt(dadd(dadd(dmul(q0, q0), dmul(q1, q1)), dmul(q2, q2)));
  if (ql == 0.0) return false;
  const double h0 = ddiv(q0, ql), h1 = ddiv(q1, ql), h2 = ddiv(q2, ql);
  const double td = dmul(2.0, h2);
  const double k0 = dsub(0.0, dmul(td, h0));
  const double k1 = dsub(0.0, dmul(td, h1));
  const double k2 = dsub(1.0, dmul(td, h2));
  const double x = dadd(dadd(dadd(0.0, dmul(g.rt[0], k0)), dmul(g.rt[1], k1)), dmul(g.rt[2], k2));
  const double y = dadd(dadd(dadd(0.0, dmul(g.rt[3], k0)), dmul(g.rt[4], k1)), dmul(g.rt[5], k2));
  const double z = dadd(dadd(dadd(0.0, dmul(g.rt[6], k0)), dmul(g.rt[7], k1)), dmul(g.rt[8], k2));
  if (z <= 0.0) return false;
  const double xp = dsub(ddiv(dmul(x, g.p2), z), g.p0);
  const double yp = dsub(ddiv(dmul(y, g.p2), z), g.p1);
  const int ix = x86_trunc_i32(dadd(ddiv(xp, g.px_x), g.cx));
  if (ix < 0 || ix > g.W - 1) return false;
  const int iy = x86_trunc_i32(dadd(ddiv(yp, g.px_y), g.cy));
  if (iy < 0 || iy > g.H - 1) return false;
  const double e = ddiv(dmul(kHcKeVnm, ql), dmul(kFourPi, -h2));
  if (e < g.elo || e > g.ehi) return false;
  ipx = ix;
  ipy = iy;
  return true;
}

template <bool kExactAll>
__global__ void dbbuild_kernel(const double *__restrict__ om, uint64_t n,
                               const int4 *__restrict__ hkl, int nh, BuildGeo g,
                               uint16_t *__restrict__ out) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int TB = blockDim.x;
  int4 *sh_hkl = reinterpret_cast<int4 *>(smem);
  float4 *sh_hklf = reinterpret_cast<float4 *>(smem + kHklChunk * sizeof(int4));
  uint32_t *sh_list = reinterpret_cast<uint32_t *>(smem + kHklChunk * 2 * sizeof(int4));
  int *sh_cnt = reinterpret_cast<int *>(sh_list + (size_t)g.S * TB);
  // per warp, the pairs that passed the screen and wait for FP64: lane << 16 | HKL
  uint32_t *q = reinterpret_cast<uint32_t *>(sh_cnt + TB) + (threadIdx.x >> 5) * (2 * 32);

  const int t = threadIdx.x;
  const int lane = t & 31;
  const unsigned lt = (1u << lane) - 1u;
  const uint64_t base = (uint64_t)blockIdx.x * TB;
  const uint64_t oid = base + t;
  const bool valid = oid < n;

  double T[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  float Tf[9];
  if (valid) {
    double m[9];
#pragma unroll
    for (int i = 0; i < 9; i++) m[i] = __ldg(om + oid * 9 + i);
    // thisOrient = OM . recip  (MatrixMultF33, LaueMatchingHeaders.h:349-357)
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
      for (int c = 0; c < 3; c++)
        T[r * 3 + c] = dadd(dadd(dmul(m[r * 3 + 0], g.recip[0 * 3 + c]),
                                 dmul(m[r * 3 + 1], g.recip[1 * 3 + c])),
                            dmul(m[r * 3 + 2], g.recip[2 * 3 + c]));
#pragma unroll
    for (int i = 0; i < 9; i++) Tf[i] = (float)T[i];
  }
  int cnt = 0;
  bool done = !valid || g.S <= 0;
  // The FP64 evaluations of the first m queued pairs (m <= 32), one per lane
  // with the owner's matrix, then their outcomes in queue order: each owner
  // takes its own in HKL order (dedup, append, stop at S) exactly as it
  // would have evaluating them one by one.
  auto evaluate = [&](int m) {
    const uint32_t ent = lane < m ? q[lane] : 0u;
    const int o = lane < m ? (int)(ent >> 16) : lane;
    double To[9];
#pragma unroll
    for (int j = 0; j < 9; j++) To[j] = __shfl_sync(0xffffffffu, T[j], o);
    int ix = 0, iy = 0;
    const bool ok = lane < m && exact_spot(To, sh_hkl[ent & 0xFFFFu], g, ix, iy);
    const uint32_t key = (uint32_t)(ix & 0xFFFF) | ((uint32_t)(iy & 0xFFFF) << 16);
    const unsigned okm = __ballot_sync(0xffffffffu, ok);
    for (int e = 0; e < m; e++) {
      const int oe = __shfl_sync(0xffffffffu, o, e);
      const uint32_t ke = __shfl_sync(0xffffffffu, key, e);
      if (lane == oe && ((okm >> e) & 1u) && !done) {
        bool dup = false;
        for (int s = 0; s < cnt; s++) dup |= (sh_list[(size_t)s * TB + t] == ke);
        if (!dup) {
          sh_list[(size_t)cnt * TB + t] = ke;
          done = (++cnt == g.S);
        }
      }
    }
    __syncwarp();
  };
  for (int c0 = 0; c0 < nh; c0 += kHklChunk) {
    const int cn = min(kHklChunk, nh - c0);
    __syncthreads();
    for (int i = t; i < cn; i += TB) {
      const int4 v = hkl[c0 + i];
      sh_hkl[i] = v;
      sh_hklf[i] = make_float4((float)v.x, (float)v.y, (float)v.z, 0.f);
    }
    __syncthreads();
    // Warp-uniform loop over the chunk: every lane screens its orientation
    // against HKL i in FP32; the pairs that pass join the warp's queue in
    // HKL order, and every 32 of them are evaluated in FP64 on all lanes at
    // once (a lane that has reached S spots queues nothing more; pairs it
    // queued before its last spot are evaluated and dropped).
    int qn = 0;
    for (int i = 0; i < cn; i++) {
      bool go = !done;
      if (!kExactAll && go) go = screen(Tf, sh_hklf[i], g);
      const unsigned bm = __ballot_sync(0xffffffffu, go);
      if (bm) {
        if (go) q[qn + __popc(bm & lt)] = ((uint32_t)lane << 16) | (uint32_t)i;
        qn += __popc(bm);
        if (qn >= 32) {
          __syncwarp();
          evaluate(32);
          const int rest = qn - 32;  // < 32: move the tail to the front
          const uint32_t v = lane < rest ? q[32 + lane] : 0u;
          __syncwarp();
          if (lane < rest) q[lane] = v;
          __syncwarp();
          qn = rest;
        }
      }
    }
    if (qn) {  // the chunk's last pairs, before its HKLs leave shared memory
      __syncwarp();
      evaluate(qn);
    }
    if (__syncthreads_and(done)) break;
  }
  sh_cnt[t] = cnt;
  __syncthreads();
  // Coalesced store of this block's records: [count, x0, y0, ...] zero padded.
  if (base >= n) return;
  const uint32_t nvalid = (uint32_t)min((uint64_t)TB, n - base);
  const uint32_t R = (uint32_t)g.R;
  const uint32_t total = nvalid * R;
  uint16_t *dst = out + base * R;
  for (uint32_t w = t; w < total; w += TB) {
    const uint32_t o = w / R, f = w - o * R;
    uint16_t v = 0;
    if (f == 0) {
      v = (uint16_t)sh_cnt[o];
    } else {
      const uint32_t s = (f - 1) >> 1;
      if ((int)s < sh_cnt[o]) {
        const uint32_t key = sh_list[(size_t)s * TB + o];
        v = (f & 1) ? (uint16_t)(key & 0xFFFF) : (uint16_t)(key >> 16);
      }
    }
    dst[w] = v;
  }
}

// Synthetic orientations: Shoemake's uniform rotations from a counter-based
// generator (SplitMix64 finaliser of counter*golden + seed*constant), the
// same uniforms as lauematching_b200/synth.py.
__device__ __forceinline__ double u01(uint64_t seed, uint64_t c) {
  uint64_t z = c * 0x9E3779B97F4A7C15ull + seed * 0xD1B54A32D192ED03ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

// Symmetry quaternions (w, x, y, z), normalised, of a fundamental-zone
// reduction of the synthetic orientations (nsym = 0: none).
struct SynthSym {
  int nsym;
  double q[24][4];
};

__global__ void synth_orient_kernel(uint64_t seed, uint64_t first, uint64_t n,
                                    double *__restrict__ out, const SynthSym sym) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t id = first + i;
    const double u1 = u01(seed, id * 3 + 0), u2 = u01(seed, id * 3 + 1),
                 u3 = u01(seed, id * 3 + 2);
    const double a = sqrt(1.0 - u1), b = sqrt(u1);
    double s2, c2, s3, c3;
    sincospi(2.0 * u2, &s2, &c2);
    sincospi(2.0 * u3, &s3, &c3);
    double x = a * s2, y = a * c2, z = b * s3, w = b * c3;
    if (sym.nsym > 0) {
      // of the equivalent rotations r (x) q keep the one with the largest
      // |scalar part| (the first such), scalar part made non-negative and
      // renormalised: the operator order and product of
      // LaueMatchingHeaders.h:111-122,166-178, as synth.hexagonal_fundamental_zone
      int best = 0;
      double bw = -1.0;
      for (int k = 0; k < sym.nsym; k++) {
        const double *r = sym.q[k];
        const double wk = fabs(r[0] * w - r[1] * x - r[2] * y - r[3] * z);
        if (wk > bw) {
          bw = wk;
          best = k;
        }
      }
      const double *r = sym.q[best];
      double Q0 = r[0] * w - r[1] * x - r[2] * y - r[3] * z;
      double Q1 = r[1] * w + r[0] * x + r[3] * y - r[2] * z;
      double Q2 = r[2] * w + r[0] * y + r[1] * z - r[3] * x;
      double Q3 = r[3] * w + r[0] * z + r[2] * x - r[1] * y;
      const double sg = Q0 < 0 ? -1.0 : 1.0;
      const double inv = sg / sqrt(Q0 * Q0 + Q1 * Q1 + Q2 * Q2 + Q3 * Q3);
      w = Q0 * inv;
      x = Q1 * inv;
      y = Q2 * inv;
      z = Q3 * inv;
    }
    double *o = out + i * 9;
    o[0] = 1.0 - 2.0 * (y * y + z * z);
    o[1] = 2.0 * (x * y - z * w);
    o[2] = 2.0 * (x * z + y * w);
    o[3] = 2.0 * (x * y + z * w);
    o[4] = 1.0 - 2.0 * (x * x + z * z);
    o[5] = 2.0 * (y * z - x * w);
    o[6] = 2.0 * (x * z - y * w);
    o[7] = 2.0 * (y * z + x * w);
    o[8] = 1.0 - 2.0 * (x * x + y * y);
  }
}

static BuildGeo make_build_geo(const lmb_geometry &geo) {
  BuildGeo g;
  for (int i = 0; i < 9; i++) {
    g.recip[i] = geo.recip[i];
    g.rt[i] = geo.rot_t[i];
    g.rtf[i] = (float)geo.rot_t[i];
  }
  g.p0 = geo.p[0];
  g.p1 = geo.p[1];
  g.p2 = geo.p[2];
  g.px_x = geo.px_x;
  g.px_y = geo.px_y;
  g.cx = 0.5 * (geo.nr_px_x - 1);
  g.cy = 0.5 * (geo.nr_px_y - 1);
  g.elo = geo.elo;
  g.ehi = geo.ehi;
  g.W = geo.nr_px_x;
  g.H = geo.nr_px_y;
  g.S = geo.max_nr_spots;
  g.R = 1 + 2 * geo.max_nr_spots;
  g.p0f = (float)g.p0;
  g.p1f = (float)g.p1;
  g.p2f = (float)g.p2;
  g.inv_pxxf = (float)(1.0 / g.px_x);
  g.inv_pyf = (float)(1.0 / g.px_y);
  g.cxf = (float)g.cx;
  g.cyf = (float)g.cy;
  g.elof = (float)g.elo;
  g.ehif = (float)g.ehi;
  g.hc4pif = (float)(kHcKeVnm / kFourPi);
  g.tolx = (float)(1e-4 * std::fabs(g.p2 / g.px_x));
  g.toly = (float)(1e-4 * std::fabs(g.p2 / g.px_y));
  return g;
}

// The FP32 screen is only sound when every geometry value is finite and
// within FP32 range; otherwise every pair takes the FP64 path.
static bool screen_sound(const lmb_geometry &geo) {
  auto ok = [](double v) { return std::isfinite(v) && std::fabs(v) < 1e30; };
  for (int i = 0; i < 9; i++)
    if (!ok(geo.rot_t[i]) || !ok(geo.recip[i])) return false;
  for (int i = 0; i < 3; i++)
    if (!ok(geo.p[i])) return false;
  return ok(geo.px_x) && ok(geo.px_y) && geo.px_x != 0 && geo.px_y != 0 && ok(geo.elo) &&
         ok(geo.ehi) && std::fabs(geo.p[2] / geo.px_x) < 1e30 && std::fabs(geo.p[2] / geo.px_y) < 1e30;
}

// Threads per block so that the [S][TB] pixel lists fit in shared memory.
static int build_block(int S) {
  int tb = 128;
  while (tb > 32 && (size_t)S * tb * 4 > 160 * 1024) tb /= 2;
  return tb;
}

size_t dbbuild_smem_bytes(int S) {
  const int tb = build_block(S);
  // HKL chunk (int and float copies), pixel lists, counts, per-warp queues of 64
  return kHklChunk * 2 * sizeof(int4) + (size_t)S * tb * 4 + (size_t)tb * 4 + (size_t)tb * 8;
}

int dbbuild_launch(const double *d_om, uint64_t n, const int4 *d_hkl, int nh,
                   const lmb_geometry &geo, uint16_t *d_out, cudaStream_t st, bool exact_all) {
  if (n == 0) return LMB_OK;
  const int S = geo.max_nr_spots;
  LMB_REQUIRE(S >= 1 && (size_t)S * 32 * 4 <= 160 * 1024,
              "MaxNrLaueSpots=%d outside the supported range 1..1280", S);
  const BuildGeo g = make_build_geo(geo);
  const bool all = exact_all || !screen_sound(geo);
  const int tb = build_block(S);
  const size_t smem = dbbuild_smem_bytes(S);
  const uint64_t blocks = (n + tb - 1) / tb;
  LMB_REQUIRE(blocks < (1ull << 31), "too many orientations (%llu)", (unsigned long long)n);
  if (all) {
    LMB_CUDA(cudaFuncSetAttribute(dbbuild_kernel<true>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dbbuild_kernel<true><<<(unsigned)blocks, tb, smem, st>>>(d_om, n, d_hkl, nh, g, d_out);
  } else {
    LMB_CUDA(cudaFuncSetAttribute(dbbuild_kernel<false>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dbbuild_kernel<false><<<(unsigned)blocks, tb, smem, st>>>(d_om, n, d_hkl, nh, g, d_out);
  }
  LMB_CUDA(cudaGetLastError());
  return LMB_OK;
}

// The 12 operators of the hexagonal (622) group, LaueMatchingHeaders.h:111-122
// (5-decimal values, normalised here).
static const double kHexSym[12][4] = {
    {1, 0, 0, 0},          {0.86603, 0, 0, 0.5},  {0.5, 0, 0, 0.86603},  {0, 0, 0, 1},
    {0.5, 0, 0, -0.86603}, {0.86603, 0, 0, -0.5}, {0, 1, 0, 0},          {0, 0.86603, 0.5, 0},
    {0, 0.5, 0.86603, 0},  {0, 0, 1, 0},          {0, -0.5, 0.86603, 0}, {0, -0.86603, 0.5, 0}};

int synth_orient_launch(uint64_t seed, uint64_t first, uint64_t n, double *d_out,
                        cudaStream_t st, uint32_t flags) {
  if (n == 0) return LMB_OK;
  SynthSym sym{};
  if (flags & LMB_BUILD_SYNTH_HEX_FZ) {
    sym.nsym = 12;
    for (int k = 0; k < 12; k++) {
      const double *q = kHexSym[k];
      const double nrm = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
      for (int j = 0; j < 4; j++) sym.q[k][j] = q[j] / nrm;
    }
  }
  const uint64_t blocks = std::min<uint64_t>((n + 255) / 256, 148ull * 32);
  synth_orient_kernel<<<(unsigned)blocks, 256, 0, st>>>(seed, first, n, d_out, sym);
  LMB_CUDA(cudaGetLastError());
  return LMB_OK;
}

}  // namespace lmb
