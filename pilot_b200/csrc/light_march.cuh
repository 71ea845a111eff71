// light_march.cuh — one light ray of the map build: the march of
// TransmittanceMapGenerator::operator() (beams/rendering/TransmittanceMap.h:279-332)
// from the light towards a map vertex (one sample at a time, or two deep in the
// exact form's skipping march). Shared by K1 (k_exact.cu), the batched kernel
// (k_batch.cu) and the learned form's probe check (k_mlp_probe.cu).
// Compiled with -fmad=false (see exact_device.cuh).
#pragma once
#include <cuda_fp16.h>

#include <type_traits>

#include "exact_device.cuh"

namespace beams {

// Opacity accumulation of one light ray.
// Exact form: o <- o + (1 - o) a (TransmittanceMap.h:329-330); o == 1 is a fixed point.
// Precision form: optical depth tau += -ln(1 - a) in float with Kahan
// compensation over the non-zero terms (the per-entry -ln(1 - a) comes from a
// table), a = 1 cuts the ray, and the map stores the transmittance exp(-tau) as
// binary16. In both forms a sample of alpha 0 leaves the state unchanged, which
// is what lets the march skip empty macro-cells.
template <bool PREC> struct Accum;
template <> struct Accum<false> {
  float o;
  __device__ __forceinline__ void init(float o0) { o = o0; }
  __device__ __forceinline__ bool add(const float* s_a, const float*, int idx) {
    o = o + (1.f - o) * s_a[idx];
    return o == 1.f;
  }
  __device__ __forceinline__ void store(void* map, int id) const { ((float*)map)[id] = o; }
};
template <> struct Accum<true> {
  float sum, comp;
  bool cut;
  __device__ __forceinline__ void init(float) {
    sum = 0.f;
    comp = 0.f;
    cut = false;
  }
  __device__ __forceinline__ bool add(const float*, const float* s_tau, int idx) {
    const float ti = s_tau[idx];
    if (ti == __int_as_float(0x7f800000)) {
      cut = true;
      return true;
    }
    if (ti == 0.f) return false;  // alpha 0 adds nothing (no compensation step either)
    const float y = ti - comp;
    const float t = sum + y;
    comp = (t - sum) - y;
    sum = t;
    return sum >= 18.f;  // exp(-18) < 2^-25: the binary16 result is 0 from here on
  }
  __device__ __forceinline__ void store(void* map, int id) const {
    const float tr = cut ? 0.f : (float)exp(-(double)sum);
    ((__half*)map)[id] = __float2half_rn(tr);
  }
};

// March from L towards vertex V. prefix(dir) gives the starting opacity (0,
// or the cross-brick prefix of the multi-brick Phase 3). ns counts the samples
// marched. With SKIP, occ is the macro-cell occupancy (see occupied()).
// PIPE: sample k+1 is located and its loads issued before sample k is
// composited (two samples' loads in flight per ray). That pays only in the
// exact form's skipping march; elsewhere the march issues one sample at a time,
// which needs fewer registers and instructions (the 257^3-vertex map of a
// 512^3 noise field went 2.97 -> 2.78 ms at 4 blocks per SM, 2.70 ms at 6).
template <typename QuadT, bool PREC, bool SKIP, bool RECT = false, bool PIPE = SKIP && !PREC, bool REG_CONSTS = PREC,
          typename Prefix>
__device__ __forceinline__ void march_vertex(const ExactGeo& g, const QuadT* __restrict__ quads, const float4* T0,
                                             const float4* T1, const float4* T2, const float* s_a,
                                             const float* s_tau, const unsigned char* __restrict__ occ,
                                             const float V[3], const float L[3], Prefix prefix, Accum<PREC>& acc,
                                             unsigned& ns) {
  const int cm0 = g.n[0] - 2, cm1 = g.n[1] - 2, cm2 = g.n[2] - 2;
  // Loop constants: with REG_CONSTS derived here (held in registers), else read
  // at each use from g's loop-constant fields, which in a kernel's parameter
  // block cost no registers (the exact light march: 2.59 -> 2.38 ms at six
  // blocks per SM). The precision march (1.5% faster so) and the batch kernel,
  // whose geometry lives in shared memory, derive them.
  unsigned qx, qz;  // FieldF32, and quads with REG_CONSTS
  QuadLoad<QuadT>::strides(g, qx, qz);
  const int n1 = g.tf_n - 1;
  const float v[3] = {V[0] - L[0], V[1] - L[1], V[2] - L[2]};
  const float rs = 1.f / sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  const float dir[3] = {v[0] * rs, v[1] * rs, v[2] * rs};
  float tmin, tmax;
  segment_aabb(g, L, V, tmin, tmax);
  const float st[3] = {L[0] + tmin * dir[0], L[1] + tmin * dir[1], L[2] + tmin * dir[2]};
  float s[3] = {st[0], st[1], st[2]};
  const float len2 = (tmax - tmin) * (tmax - tmin);
  const float sdx = g.step * dir[0], sdy = g.step * dir[1], sdz = g.step * dir[2];
  // The sample positions do not depend on the opacity, so with PIPE sample
  // k+1 is located and its loads issued before sample k is composited. The
  // break conditions are evaluated in the reference's order for every sample;
  // only o == 1 ends the march early, after which a prefetched sample is
  // discarded.
  // Empty macro-cells (occ == 0: every value there has TF alpha 0) are
  // stepped over without a field fetch: such a sample leaves the state
  // unchanged (Accum), so only its position update and break checks run. sk
  // counts the samples skipped before the one returned; they are counted as
  // marched once that sample is composited (or the ray ends on its own).
  int b = g.light_budget;
  // The first `fast` iterations are certain to pass the budget and distance
  // tests, so they skip them. With u = 2^-24, after k steps the float position
  // lies within k (step (1 + 4u) + 2 sqrt(3) u M) of the start (M bounds every
  // |coordinate| on the segment), so |s - st|^2 <= len2 holds, rounding
  // included, while k < (1 - 4u) (tmax - tmin) / (that per-step bound); the
  // constants below double each u term, and two more steps are kept back.
  int fast = 0;
  {
    const float dl = tmax - tmin;
    if (dl > 0.f) {
      const float M = fmaxf(fmaxf(fabsf(st[0]), fabsf(st[1])), fabsf(st[2])) + dl + g.step;
      const float kf = (dl * 0.99999f) / (g.step * 1.00001f + 4e-7f * M);
      if (kf > 2.f) fast = min((int)fminf(kf, 1e9f) - 2, b);
    }
  }
  b -= fast;
  auto gen = [&](float v8[8], float pc[3], unsigned& sk) -> bool {
    sk = 0;
    for (;;) {
      if (fast > 0) {
        --fast;
      } else {
        if (b-- <= 0) return false;
        const float q0 = s[0] - st[0], q1 = s[1] - st[1], q2 = s[2] - st[2];
        if (!(q0 * q0 + q1 * q1 + q2 * q2 <= len2)) return false;
      }
      s[0] = s[0] + sdx;
      s[1] = s[1] + sdy;
      s[2] = s[2] + sdz;
      if (!inside_vol(g, s)) return false;
      if (SKIP && !occupied(g, occ, s)) {
        ++sk;
        continue;
      }
      float4 e0, e1, e2;
      int c0, c1, c2;
      if constexpr (RECT) {
        c0 = find_cell_bsearch_rect(T0, cm0, s[0], e0);
        c1 = find_cell_bsearch_rect(T1, cm1, s[1], e1);
        c2 = find_cell_bsearch_rect(T2, cm2, s[2], e2);
      } else {
        // s is inside the volume (tested above), so s - org >= 0 exactly and the
        // seeded guesses need no lower clamp. A guess is the found cell unless s
        // lies within an ulp of a cell face: one branch tests the three axes and
        // the rare walk runs out of line, so the common path carries none of its
        // code (the 257^3-vertex map of a 512^3 noise field: 2.66 -> 2.59 ms;
        // the same walks inline behind one branch ran 2.75 ms, and three
        // separate per-axis branches 2.66 ms)
        c0 = trunc_small(fminf((s[0] - g.org[0]) * g.invh[0], REG_CONSTS ? (float)cm0 : g.cmaxf[0]));
        c1 = trunc_small(fminf((s[1] - g.org[1]) * g.invh[1], REG_CONSTS ? (float)cm1 : g.cmaxf[1]));
        c2 = trunc_small(fminf((s[2] - g.org[2]) * g.invh[2], REG_CONSTS ? (float)cm2 : g.cmaxf[2]));
        e0 = T0[c0];
        e1 = T1[c1];
        e2 = T2[c2];
        if ((s[0] <= e0.x) | (s[0] > e0.y) | (s[1] <= e1.x) | (s[1] > e1.y) | (s[2] <= e2.x) | (s[2] > e2.y)) {
          if constexpr (PREC) {
            // the precision march keeps the walks inline (out of line its
            // 640^3 skipping build ran 1.5% slower)
            while (c0 > 0 && s[0] <= e0.x) e0 = T0[--c0];
            while (c0 < cm0 && s[0] > e0.y) e0 = T0[++c0];
            while (c1 > 0 && s[1] <= e1.x) e1 = T1[--c1];
            while (c1 < cm1 && s[1] > e1.y) e1 = T1[++c1];
            while (c2 > 0 && s[2] <= e2.x) e2 = T2[--c2];
            while (c2 < cm2 && s[2] > e2.y) e2 = T2[++c2];
          } else {
            const int3 cc = walk_cells_bsearch(T0, T1, T2, cm0, cm1, cm2, s[0], s[1], s[2], c0, c1, c2);
            c0 = cc.x;
            c1 = cc.y;
            c2 = cc.z;
            e0 = T0[c0];
            e1 = T1[c1];
            e2 = T2[c2];
          }
        }
      }
      if constexpr (REG_CONSTS || std::is_same<QuadT, FieldF32>::value)
        QuadLoad<QuadT>::cell(quads, (unsigned)c2 * qz + (unsigned)c1 * qx + (unsigned)c0, qx, qz, v8);
      else  // the quad strides straight from the parameter space
        QuadLoad<QuadT>::cell(quads, (unsigned)c2 * g.qzs + (unsigned)c1 * g.qxs + (unsigned)c0, g.qxs, g.qzs, v8);
      // pcoords = (p - min) / (max - min) (RectilinearMeshOracle.h:189-192)
      pc[0] = div_rn_markstein(s[0] - e0.x, e0.z, e0.w);
      pc[1] = div_rn_markstein(s[1] - e1.x, e1.z, e1.w);
      pc[2] = div_rn_markstein(s[2] - e2.x, e2.z, e2.w);
      return true;
    }
  };
  // TF index of a normalised scalar (TransmittanceMap.h:322-326)
  auto tf_idx = [&](float scalar) {
    return REG_CONSTS ? tf_index_clamped(scalar * (float)n1, n1) : tf_index_clamped_f(scalar * g.n1f, g.n1f);
  };
  acc.init(prefix(dir));
  float va[8], pa[3];
  unsigned ska;
  if constexpr (!PIPE) {
    // Every gen() call takes one step (fast or b), so the samples marched are
    // the steps taken less a failing last one: the precision march counts them
    // so at the end (its 640^3 build 6.06 -> 5.96 ms); the exact march counts
    // per sample, which runs faster there (2.38 against 2.42 ms).
    const int steps0 = fast + b;
    for (;;) {
      if (!gen(va, pa, ska)) {
        if constexpr (PREC) ns += (unsigned)(steps0 - (fast + b) - 1);
        else ns += ska;  // skipped samples before the end of the ray
        break;
      }
      float scalar = hex_interp(va, pa[0], pa[1], pa[2]);
      scalar = (scalar - g.min_scalar) * g.inv_delta;
      if constexpr (!PREC) ns += 1 + ska;
      // Stop when the accumulated value can no longer change (see Accum).
      if (acc.add(s_a, s_tau, tf_idx(scalar))) {
        if constexpr (PREC) ns += (unsigned)(steps0 - (fast + b));
        break;
      }
    }
    return;
  }
  static_assert(!PIPE || SKIP, "the two-sample pipeline is written for the skipping march");
  float vb[8], pb[3];
  unsigned skb;
  bool ok = gen(va, pa, ska);
  if (!ok) ns += ska;
  while (ok) {
    const bool okb = gen(vb, pb, skb);
    bool done;
    {
      float scalar = hex_interp(va, pa[0], pa[1], pa[2]);
      scalar = (scalar - g.min_scalar) * g.inv_delta;
      done = acc.add(s_a, s_tau, tf_idx(scalar));
      ns += 1 + ska;
    }
    // Stop when the accumulated value can no longer change (see Accum).
    if (done) break;
    if (!okb) {
      ns += skb;
      break;
    }
    ok = gen(va, pa, ska);
    {
      float scalar = hex_interp(vb, pb[0], pb[1], pb[2]);
      scalar = (scalar - g.min_scalar) * g.inv_delta;
      done = acc.add(s_a, s_tau, tf_idx(scalar));
      ns += 1 + skb;
    }
    if (done) break;
    if (!ok) ns += ska;
  }
}

}  // namespace beams
