// The null-path forward tracer (--algo pt2, renderingalgorithms_pathtracing2.cxx), split
// into the same wavefront stages as the plain tracer.  Included by tt_kernels.cu after the
// traversal, light and queue helpers.
//
// Differences from the plain tracer that the stages below implement:
//   - distance sampling by hero-wavelength delta tracking with null collisions
//     (nullpath::Tracking, media_integrator.cxx:240-286, 330-378) inside the shade stage; a
//     vacuum segment draws one uniform, as the reference's tracker does with a zero majorant;
//   - the path carries 3 x 3 matrices of per-wavelength distance-pdf ratios
//     (weights_track, and weights_track_then_null for the last segment) that enter the MIS
//     weights, a balance heuristic over the hero wavelengths (MisWeight, :452-476);
//   - next-event estimation only at scatter vertices (none at the camera), with the light
//     picked by TowerSampling over the light types and bisection over a uniform CMF
//     (LightSelectionProbabilityMap); the shadow ray's transmission is a null-path
//     estimate (nullpath::Transmission, media_integrator.cxx:288-325, 384-420);
//   - no Russian roulette: a path ends when its node count (starting at 2) exceeds
//     max_ray_depth (RayTermination, rendering_util.hxx:383-412);
//   - path regularisation: after a rough bounce the dielectric is mollified and microfacet
//     lobes are widened to the largest roughness met so far (SampleScatterer, :563-573).
//
// Deviation, kept by the oracle too: the shadow ray's transmission estimate draws from its
// own stream, seeded from the path's random state at the connection (the reference draws
// from the path's sampler, which the wavefront has moved on from by the time the shadow
// ray is traced).  A path whose weights vanished stops at once (the reference walks it to
// the depth limit adding nothing).

// nullpath::Spectral33: row i = the wavelength whose distance sampling produced the path,
// column j = the pdf of that path under wavelength j's sampling, as ratios.
struct M33f {
  float a[9];
};
__device__ __forceinline__ float fix_nan(float x) { return isnan(x) ? INFINITY : x; }
__device__ __forceinline__ void m33_ones(M33f& m) {
#pragma unroll
  for (int k = 0; k < 9; ++k) m.a[k] = 1.f;
}
// AccumulateContributions(w, x) (media_integrator.cxx:223-229).
__device__ __forceinline__ void m33_acc(M33f& w, const M33f& x) {
#pragma unroll
  for (int k = 0; k < 9; ++k) w.a[k] = fix_nan(w.a[k] * x.a[k]);
}
// AccumulateContributions(w, f, p) (:231-238): w_ij *= p_j / f_i.
__device__ __forceinline__ void m33_acc(M33f& w, float3 f, float3 p) {
  const float fi[3] = {f.x, f.y, f.z}, pj[3] = {p.x, p.y, p.z};
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) w.a[3 * i + j] = fix_nan(w.a[3 * i + j] * fix_nan((1.f / fi[i]) * pj[j]));
}
__device__ __forceinline__ float3 m33_row_mean(const M33f& m) {
  return f3((m.a[0] + m.a[1] + m.a[2]) * (1.f / 3.f), (m.a[3] + m.a[4] + m.a[5]) * (1.f / 3.f),
            (m.a[6] + m.a[7] + m.a[8]) * (1.f / 3.f));
}
__device__ __forceinline__ float3 m33_row_mean_scaled(const M33f& m, float s) {
  M33f t;
#pragma unroll
  for (int k = 0; k < 9; ++k) t.a[k] = fix_nan(m.a[k] * s);
  return m33_row_mean(t);
}
__device__ __forceinline__ float3 div3(float3 a, float3 b) { return f3(a.x / b.x, a.y / b.y, a.z / b.z); }

// Extinction majorant of a segment and the coefficients at a point (Medium::
// ComputeMajorante, EvaluateCoeffs); medium -1 is the vacuum.
__device__ __forceinline__ float3 majorant2(const DevScene& sc, int medium, float3 org, float3 dir, float len,
                                            Lambda l) {
  if (medium < 0) return f3(0.f, 0.f, 0.f);
  const DevMedium& M = sc.media[medium];
  if (M.kind == TT_MEDIUM_ATMOSPHERE) {
    const float m = atm_segment_majorant(M, org, dir, len);
    return f3(m, m, m);
  }
  return take(M.sigma_ext, l);
}
__device__ __forceinline__ void coeffs2(const DevScene& sc, int medium, float3 pos, Lambda l, float3* ss, float3* st) {
  if (medium < 0) {
    *ss = *st = f3(0.f, 0.f, 0.f);
    return;
  }
  const DevMedium& M = sc.media[medium];
  if (M.kind == TT_MEDIUM_ATMOSPHERE) {
    atm_coeffs(M, atm_altitude(M, pos), l, ss, st);
    return;
  }
  *ss = take(M.sigma_s, l);
  *st = take(M.sigma_ext, l);
}
__device__ __forceinline__ float3 exp_maj(float3 maj, float x) {
  return f3(expf(-x * maj.x), expf(-x * maj.y), expf(-x * maj.z));
}

// nullpath::Tracking on one segment: hero-wavelength delta tracking.  Returns true at a
// real collision, at distance *t_out.  At most 10^4 steps (then no collision).
template <class R>
__device__ __forceinline__ bool track_segment2(const DevScene& sc, int medium, float3 org, float3 dir, float len,
                                               M33f& ft, M33f& fn, R& rng, Lambda l, float* t_out) {
  const float3 maj = majorant2(sc, medium, org, dir, len, l);
  const float mfp = 1.f / maj.x;
  float t = 0.f;
  for (int it = 1; it < 10000; ++it) {
    const float tlocal = fminf(kLargeNumber, -logf(1.f - rng.uniform()) * mfp);
    const float3 tr = exp_maj(maj, fminf(tlocal, len - t));
    t += tlocal;
    if (t >= len) {
      m33_acc(ft, tr, tr);
      m33_acc(fn, tr, tr);
      return false;
    }
    float3 ss, st;
    coeffs2(sc, medium, org + dir * t, l, &ss, &st);
    const float3 sn = maj - st;
    const float prob_n = sn.x * mfp;
    if (rng.uniform() < prob_n) {
      m33_acc(ft, mul(tr, sn), mul(tr, sn));
      m33_acc(fn, mul(tr, sn), mul(tr, maj));
    } else {
      m33_acc(ft, mul(tr, st), mul(tr, st));
      m33_acc(fn, mul(tr, st), tr);
      *t_out = t;
      return true;
    }
  }
  return false;
}

// nullpath::Transmission on one segment: every collision is a null collision.  Stops once
// every diagonal entry of the null matrix exceeds LargeNumber (the estimate is zero).
template <class R>
__device__ __forceinline__ void transmit_segment2(const DevScene& sc, int medium, float3 org, float3 dir, float len,
                                                  M33f& ft, M33f& fn, R& rng, Lambda l) {
  const float3 maj = majorant2(sc, medium, org, dir, len, l);
  const float mfp = 1.f / maj.x;
  M33f st_, sn_;
  m33_ones(st_);
  m33_ones(sn_);
  float t = 0.f;
  for (int it = 1; it < 10000; ++it) {
    const float tlocal = fminf(kLargeNumber, -logf(1.f - rng.uniform()) * mfp);
    const float3 tr = exp_maj(maj, fminf(tlocal, len - t));
    t += tlocal;
    if (t >= len) {
      m33_acc(st_, tr, tr);
      m33_acc(sn_, tr, tr);
      break;
    }
    float3 ss, st;
    coeffs2(sc, medium, org + dir * t, l, &ss, &st);
    const float3 sn = maj - st;
    m33_acc(st_, mul(tr, sn), mul(tr, sn));
    m33_acc(sn_, mul(tr, sn), mul(tr, maj));
    if (sn_.a[0] > kLargeNumber && sn_.a[4] > kLargeNumber && sn_.a[8] > kLargeNumber) {
#pragma unroll
      for (int k = 0; k < 9; ++k) sn_.a[k] = INFINITY;
      break;
    }
  }
  m33_acc(ft, st_);
  m33_acc(fn, sn_);
}

// MisWeight(scatter_pdf, pdf_other, d, d_other) applied to a contribution x: x * w / den
// with (w, den) = (1, row mean of d) when there is no MIS, else (pdf, row means of d * pdf
// plus d_other * pdf_other).  Without media both matrices are all ones.
template <bool MEDIA>
__device__ __forceinline__ float3 mis2(const DevScene& sc, float3 x, bool has_pdf, float pdf, bool delta,
                                       float pdf_other, const M33f& d, const M33f& d_other) {
  if (!has_pdf || delta || !(sc.sample_bsdf && sc.sample_lights)) return MEDIA ? div3(x, m33_row_mean(d)) : x;
  if (MEDIA) return div3(x * pdf, m33_row_mean_scaled(d, pdf) + m33_row_mean_scaled(d_other, pdf_other));
  const float den = fix_nan(pdf) + fix_nan(pdf_other);
  return x * (pdf / den);
}

// AddDirectLighting (renderingalgorithms_pathtracing2.cxx:479-560) up to the shadow ray:
// light pick, connection segment (offset at the eye end only, Lights::Detail::
// SegmentToPoint / SegmentToEnv, light.cxx:218-266), light weight, scatter factor at the
// eye.  The light pdf returned for MIS is the light's own density (solid angle), without
// the selection probability, as in the reference.  `s` is null at a volume vertex.
template <bool MEDIA>
__device__ __forceinline__ void nee2(const DevScene& sc, const PathState& p, int qbounce, int slot, Smp2& rng, Lambda l,
                                     float3 beta, float3 wi, const Surf* s, float rough, int vmed, float3 vpos,
                                     const MTracker& mt, const M33f& wt) {
  if (sc.num_env == 0 && sc.num_area_lights == 0 && sc.num_point_lights == 0) return;  // no light to pick
  const int which = tower_sampling4(sc.type_probs, rng.uniform());
  const int nl = which == LIGHT_ENV ? 1 : (which == LIGHT_AREA ? sc.num_area_lights : sc.num_point_lights);
  // TowerSamplingBisection over the uniform CMF (k + 1) / nl.
  const float rr = rng.uniform();
  int li = min(nl - 1, max(0, (int)(rr * (float)nl)));
  if (li > 0 && rr < (float)li / (float)nl) --li;
  if (li < nl - 1 && rr >= (float)(li + 1) / (float)nl) ++li;
  const float prob = sc.type_probs[which] / (float)nl;
  const float3 pos0 = s ? s->pos : vpos;
  float3 org = pos0, dir;
  float len, pdf;
  bool delta = false;
  float3 light_weight;
  if (which == LIGHT_ENV) {
    const int i = rng.uniform_int(0, sc.num_env - 1);
    DirSample e = env_sample_one(sc.env[i], rng, l);
    e.pdf *= 1.f / (float)sc.num_env;
    dir = -e.dir;
    len = sc.long_distance;
    if (s) org = org + offset_at(*s, dir);
    pdf = e.pdf;
    delta = e.delta;
    light_weight = e.value * (1.f / (e.pdf * prob));
  } else {
    float3 lpos, lng = f3(0.f, 0.f, 1.f), lns = lng;
    float area_pdf = 1.f;
    int lprim = -1;
    if (which == LIGHT_AREA) {
      float r[2];
      rng.square(r);
      const float4 a = __ldg(&sc.area_verts[3 * li]);
      const float4 b = __ldg(&sc.area_verts[3 * li + 1]);
      const float4 c = __ldg(&sc.area_verts[3 * li + 2]);
      lprim = __ldg(&sc.area_lights[li]);
      if (a.w != 0.f) {
        const float3 off = to_uniform_sphere(r) * b.x;
        lpos = xyz(a) + off;
        lng = normalize3(off);
        lns = lng;
        area_pdf = 1.f / (b.x * b.x * 4.f * kPi);
      } else {
        const float3 w = to_triangle_barycentric(r);
        const float3 p0 = xyz(a), p1 = xyz(b), p2 = xyz(c);
        lpos = p0 * w.x + p1 * w.y + p2 * w.z;
        lng = normalize3(cross3(p1 - p0, p2 - p0));
        lns = lng;
        if (sc.normals) {
          const uint4 ti = __ldg(&sc.tri_idx[lprim]);
          const float* N = sc.normals;
          lns = normalize3(f3(N[3 * ti.x], N[3 * ti.x + 1], N[3 * ti.x + 2]) * w.x +
                           f3(N[3 * ti.y], N[3 * ti.y + 1], N[3 * ti.y + 2]) * w.y +
                           f3(N[3 * ti.z], N[3 * ti.z + 1], N[3 * ti.z + 2]) * w.z);
        }
        area_pdf = 1.f / tri_area(p0, p1, p2);
      }
    } else {
      const float* pl = sc.point_lights + (size_t)li * (NBINS + 3);
      lpos = f3(pl[NBINS], pl[NBINS + 1], pl[NBINS + 2]);
      delta = true;
    }
    const float3 dd = lpos - org;
    len = len3(dd);
    if (len > 0.f) {
      dir = dd * (1.f / len);
    } else {
      len = kEps;
      dir = s ? s->n : f3(1.f, 0.f, 0.f);
    }
    if (s) org = org + offset_at(*s, dir);
    float3 val;
    if (which == LIGHT_AREA) {
      const DevMaterial& lm = sc.materials[__ldg(&sc.tri_idx[lprim]).w];
      const float vis = dot3(lng, -dir) > 0.f ? 1.f : 0.f;
      val = take(lm.emission, l) * (vis / (2.f * kPi) * fabsf(dot3(lns, dir)));
      pdf = len * len / fabsf(dot3(dir, lng) + kEps) * area_pdf;
    } else {
      const float* pl = sc.point_lights + (size_t)li * (NBINS + 3);
      val = take(pl, l) * (1.f / (4.f * kPi));
      pdf = len * len / kEps;
    }
    light_weight = val * (1.f / (area_pdf * prob) / (len * len));
  }
  // Scatter factor at the eye.
  float3 pw = beta;
  float bsdf_pdf = 0.f;
  MTracker smt = mt;
  if (s) {
    const DevMaterial& m = sc.materials[s->material];
    pw = mul(pw * fabsf(dot3(s->ns, dir)), eval_bsdf(m, wi, *s, dir, l, &bsdf_pdf, rough));
    if (MEDIA && dot3(dir, s->n) < 0.f) going_through(sc, smt, dir, s->ng, s->material);
  } else {
    const DevMedium& M = sc.media[vmed];
    float3 ss, st;
    pw = mul(pw, medium_phase_eval(M, vpos, wi, dir, l, &bsdf_pdf));
    coeffs2(sc, vmed, vpos, l, &ss, &st);
    pw = mul(pw, div3(ss, st + f3(kEps, kEps, kEps)));
  }
  const float3 pre = mul(pw, light_weight);
  if (is_zero(pre)) return;
  const bool mis_on = !delta && sc.sample_bsdf && sc.sample_lights;
  float3 contrib = pre;
  if (MEDIA) {
    p.sh_med[slot] = make_float4(mis_on ? pdf : -1.f, bsdf_pdf, __uint_as_float((unsigned)(rng.rng.state & 0xffffffffu)),
                                 __uint_as_float((unsigned)(rng.rng.state >> 32)));
    p.sh_track[slot] = store_tracker(smt);
    if (rng.mats) p.sh_qmc[slot] = rng.q;
#pragma unroll
    for (int k = 0; k < 9; ++k) p.sh_wt[9 * (size_t)slot + k] = wt.a[k];
  } else {
    M33f ones;
    m33_ones(ones);
    contrib = mis2<false>(sc, pre, true, pdf, delta, bsdf_pdf, ones, ones);
  }
  const int q = warp_append(sh_count(p, qbounce));
  p.sh_q[q] = slot;
  p.sh_o[slot] = make_float4(org.x, org.y, org.z, len * 0.9999f);
  p.sh_d[slot] = make_float4(dir.x, dir.y, dir.z, __int_as_float(-1));
  p.sh_c[slot] = make_float4(contrib.x, contrib.y, contrib.z, 0.f);
}

// One step of CameraRenderWorker::RenderPixel's loop (:410-443) for each queued path:
// tracking to the closest hit, emission with MIS, next-event estimation, scattering.
template <bool MEDIA, bool SPH, bool WIDE>
__global__ void __launch_bounds__(256) k_shade2(DevScene sc, PathState p, int bounce) {
  const int n = *ext_count(p, bounce);
  const int* q = p.ext_q[bounce & 1];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int slot = q[i];
    const float4 h = p.hit[slot];
    const float3 org = xyz(p.ray_o[slot]);
    const float3 dir = xyz(p.ray_d[slot]);
    uint4 meta = p.meta[slot];
    const Lambda l = unpack_lambda(meta.y);
    const float4 b4 = p.beta[slot];
    float3 beta = xyz(b4);
    const bool has_last = (meta.w & 2u) != 0u, last_delta = (meta.w & 1u) != 0u;
    const float last_pdf = b4.w;
    float3 acc = xyz(p.accum[slot]);
    Smp2 rng;
    rng.rng = Rng{p.rng_state[slot], p.rng_inc[slot]};
    rng.mats = sc.sobol;
    if (sc.sobol) rng.q = p.qmc[slot];
    const int tri = __float_as_int(h.w);
    bool done = false;
    M33f wt, wtn;
    MTracker mt{0xffffffffu, -1};
    bool volume = false;
    int vmed = -1;
    float3 vpos = f3(0.f, 0.f, 0.f);
    if (MEDIA) {
      // Tracking through the medium segments in front of the surface hit.
#pragma unroll
      for (int k = 0; k < 9; ++k) wt.a[k] = p.wt2[9 * (size_t)slot + k];
      mt = load_tracker(p.track[slot]);
      M33f ft, fn;
      m33_ones(ft);
      m33_ones(fn);
      const float vend = (tri >= 0 ? h.x : kLargeNumber) * 0.9999f;
      const RayPre r = prepare_ray(org, dir);
      float snear = 0.f;
      for (int k = 0;; ++k) {
        float tc;
        const int cs = next_crossing<SPH, WIDE>(sc, r, snear, vend, &tc, p.err);
        const float sfar = cs >= 0 ? tc : vend;
        float tcol;
        const int m = mt.cur;
        if (track_segment2(sc, m, org + dir * snear, dir, sfar - snear, ft, fn, rng, l, &tcol)) {
          volume = true;
          vmed = m;
          vpos = org + dir * (snear + tcol);
          break;
        }
        if (cs < 0) break;
        if (k >= kMaxCrossings) {
          atomicOr(p.err, ERR_CROSSINGS);
          done = true;
          break;
        }
        float3 ng;
        int mat;
        crossing_info(sc.vtris, cs, org, dir, sfar, &ng, &mat);
        going_through(sc, mt, dir, ng, mat);
        snear = sfar;
      }
      wtn = wt;
      m33_acc(wtn, fn);
      m33_acc(wt, ft);
    } else {
      m33_ones(wt);
      m33_ones(wtn);
      rng.uniform();  // the vacuum segment's free-flight sample
    }
    const int count0 = (int)meta.z;  // node count of this vertex
    rng.prep(((unsigned)count0 << 1) | 1u);
    const float rough = p.rough[slot];
    Surf s;
    if (!done && !volume && tri < 0) {
      // AddEnvEmission (:625-648).
      if (sc.sample_bsdf && sc.num_env > 0) {
        const float3 rad = env_eval_total(sc, -dir, l);
        const float pdf_env = env_pdf_total(sc, -dir) * sc.type_probs[0];
        acc = acc + mis2<MEDIA>(sc, mul(rad, beta), has_last, last_pdf, last_delta, pdf_env, wt, wtn);
      }
      done = true;
    }
    const float3 wi = -dir;
    if (!done && !volume) {
      const float u = h.y, v = h.z;
      const bool sphere = sc.num_spheres > 0 && is_sphere_slot(sc.tris, tri);
      s = sphere ? sphere_hit_surface(sc.tris, tri, org, dir, h.x)
                 : make_surface(sc, tri, 1.f - u - v, u, v, f3(u, v, 1.f - u - v));
      orient(s, dir);
      const DevMaterial& m = sc.materials[s.material];
      if (sc.sample_bsdf && m.emissive) {
        // MaybeAddEmission (:592-622).
        const float vis = dot3(s.ng, -dir) > 0.f ? 1.f : 0.f;
        const float3 rad = take(m.emission, l) * (vis / (2.f * kPi));
        float other = 1.f;
        if (has_last) {
          const float4 a = __ldg(&sc.tris[3 * tri]), b = __ldg(&sc.tris[3 * tri + 1]), c = __ldg(&sc.tris[3 * tri + 2]);
          const float area = __float_as_int(c.w) != 0 ? b.x * b.x * 4.f * kPi : tri_area(xyz(a), xyz(b), xyz(c));
          const float3 dd = org - s.pos;
          const float cvt = dot3(dd, dd) / fabsf(dot3(dir, s.n) + kEps);
          other = sc.type_probs[1] * sc.in_class_area * (1.f / area) * cvt;
        }
        acc = acc + mis2<MEDIA>(sc, mul(rad, beta), has_last, last_pdf, last_delta, other, wt, wtn);
      }
      if (sc.sample_lights) nee2<MEDIA>(sc, p, bounce + 1, slot, rng, l, beta, wi, &s, rough, -1, vpos, mt, wt);
    } else if (!done) {
      if (sc.sample_lights) nee2<MEDIA>(sc, p, bounce + 1, slot, rng, l, beta, wi, nullptr, rough, vmed, vpos, mt, wt);
    }
    const int count = count0 + 1;
    if (!done && count > sc.max_path_nodes - 1) done = true;
    rng.prep((unsigned)count0 << 1);
    if (!done) {
      float3 ndir, bf, norg;
      float pdf;
      bool delta = false;
      float nrough = rough;
      if (!volume) {
        const DevMaterial& m = sc.materials[s.material];
        const ScatterSample ss = sample_bsdf(m, wi, s, rng, l, rough);
        nrough = fmaxf(my_roughness(m), rough);
        pdf = ss.pdf;
        delta = ss.delta;
        ndir = ss.dir;
        bf = ss.value * (fabsf(dot3(s.ns, ss.dir)) / ss.pdf);
        norg = s.pos + offset_at(s, ss.dir);
      } else {
        const DevMedium& M = sc.media[vmed];
        float3 pval, sig_s, sig_t;
        ndir = medium_phase_sample(M, vpos, wi, rng, l, &pval, &pdf);
        coeffs2(sc, vmed, vpos, l, &sig_s, &sig_t);
        bf = mul(pval, div3(sig_s, sig_t + f3(kEps, kEps, kEps))) * (1.f / pdf);
        norg = vpos;
      }
      beta = mul(beta, bf);
      if (is_zero(beta) || !(pdf > 0.f)) {
        done = true;
      } else {
        if (MEDIA && !volume && dot3(ndir, s.n) < 0.f) going_through(sc, mt, ndir, s.ng, s.material);
        p.ray_o[slot] = make_float4(norg.x, norg.y, norg.z, 0.f);
        p.ray_d[slot] = make_float4(ndir.x, ndir.y, ndir.z, kLargeNumber);
        p.beta[slot] = make_float4(beta.x, beta.y, beta.z, pdf);
        meta.z = (unsigned)count;
        meta.w = 2u | (delta ? 1u : 0u);
        p.meta[slot] = meta;
        p.rough[slot] = nrough;
        if (MEDIA) {
          p.track[slot] = store_tracker(mt);
#pragma unroll
          for (int k = 0; k < 9; ++k) p.wt2[9 * (size_t)slot + k] = wt.a[k];
        }
        const int qe = warp_append(ext_count(p, bounce + 1));
        p.ext_q[(bounce + 1) & 1][qe] = slot;
      }
    }
    p.accum[slot] = make_float4(acc.x, acc.y, acc.z, 0.f);
    p.rng_state[slot] = rng.rng.state;
    if (sc.sobol) p.qmc[slot] = rng.q;
    if (done) {
      const int qd = warp_append(done_count(p, bounce + 1));
      p.done_q[qd] = slot;
    }
  }
}

// Shadow rays of the null-path tracer in media scenes: occlusion, then the null-path
// transmission through the medium segments on the shadow ray's own stream, then the MIS
// weight over the hero wavelengths (the end of AddDirectLighting, :537-560).  Without media
// the contribution is final at the vertex and the plain shadow kernel adds it.
template <bool SPH, bool WIDE>
__global__ void __launch_bounds__(256) k_shadow2(DevScene sc, PathState p, int bounce) {
  const int n = *sh_count(p, bounce);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int slot = p.sh_q[i];
    const float4 o = p.sh_o[slot], d = p.sh_d[slot];
    const RayPre r = prepare_ray(xyz(o), xyz(d));
    float t, b1, b2;
    TraceCounters cnt{0u, 0u};
    const int hit = trace<true, false, SPH, WIDE>(sc, r, 0.f, o.w, &t, &b1, &b2, p.err, &cnt);
    if (hit >= 0) continue;
    const Lambda l = unpack_lambda(p.meta[slot].y);
    MTracker mt = load_tracker(p.sh_track[slot]);
    const float4 med = p.sh_med[slot];
    Smp2 srng;
    srng.rng.seed_path(((unsigned long long)__float_as_uint(med.w) << 32) | __float_as_uint(med.z), p.rng_inc[slot]);
    srng.mats = sc.sobol;
    if (sc.sobol) srng.q = p.sh_qmc[slot];
    M33f ft, fn;
    m33_ones(ft);
    m33_ones(fn);
    float snear = 0.f;
    bool lost = false;
    for (int k = 0;; ++k) {
      float tc;
      const int cs = next_crossing<SPH, WIDE>(sc, r, snear, o.w, &tc, p.err);
      const float sfar = cs >= 0 ? tc : o.w;
      transmit_segment2(sc, mt.cur, xyz(o) + xyz(d) * snear, xyz(d), sfar - snear, ft, fn, srng, l);
      if (cs < 0) break;
      if (k >= kMaxCrossings) {
        atomicOr(p.err, ERR_CROSSINGS);
        lost = true;
        break;
      }
      float3 ng;
      int mat;
      crossing_info(sc.vtris, cs, xyz(o), xyz(d), sfar, &ng, &mat);
      going_through(sc, mt, xyz(d), ng, mat);
      snear = sfar;
    }
    if (lost) continue;
    M33f wt;
#pragma unroll
    for (int k = 0; k < 9; ++k) wt.a[k] = p.sh_wt[9 * (size_t)slot + k];
    m33_acc(ft, wt);
    m33_acc(fn, wt);
    const float3 c = mis2<true>(sc, xyz(p.sh_c[slot]), true, med.x, med.x < 0.f, med.y, fn, ft);
    const float4 a = p.accum[slot];
    p.accum[slot] = make_float4(a.x + c.x, a.y + c.y, a.z + c.z, 0.f);
  }
}
