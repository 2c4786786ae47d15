// The adjoint of the path tracer: gradients of an image loss with respect to every material's base
// colour and GGX alpha and every area light's power, by path replay backpropagation (Vicini,
// Speierer and Jakob, "Path Replay Backpropagation", SIGGRAPH 2021). Included by rtg_kernels.cu,
// whose sampler table and helpers it shares.
//
// A forward wave renders every path of the call and leaves each path's radiance L in its slot.
// k_adjoint_delta turns the film and the target image into the loss and, per pixel, the loss's
// derivative with respect to one path's radiance. The backward wave (k_adjoint_camera, the forward's
// k_extend, k_scan and k_scatter, then k_shade_adjoint and k_shadow_adjoint per bounce) runs every
// path again from its pixel and sample index (the sampler makes it the same path), carrying
// L_rem = L - (the contributions met so far), which is the radiance still to come. At each vertex:
// - a contribution c of area light i adds <dL, c> to light i's scale gradient, and when c is a
//   next-event estimate through the BSDF f, <dL, K * df> to the material's (c = K * f);
// - a BSDF sample scales all later radiance by f / pdf: the material's gradient gains
//   <dL, L_rem * df / f>, the pdf held fixed (detached sampling, unbiased);
// - a clear medium scales later radiance by exp(-sigma t): its base colour gains
//   <dL, L_rem * t / (base * absorption)>.
// df is the central difference of the BSDF over base colour (all three channels at once: each
// channel of f depends on its own channel of the base colour only) or over alpha, with the
// perturbed BSDFs built on the host by the same construction as the forward ones. Selection
// probabilities, MIS weights and roulette are held fixed, as detached sampling requires.
#pragma once

namespace rtg {

constexpr int MAX_ADJOINT_PARAMS = 4 * 64 + MAX_LIGHTS;


__device__ __forceinline__ Rgb rgb_sub(Rgb a, Rgb b) { return rgb(a.r - b.r, a.g - b.g, a.b - b.b); }

// The loss derivative a path uses: its pixel's, from the other half of the call's samples when the
// call has two halves (samples before A.split and from A.split on).
__device__ __forceinline__ size_t adj_dpath_index(const AdjointDev& A, const WaveDesc& w, uint32_t x, uint32_t y, uint32_t index) {
    const size_t p = (size_t)(y - w.y0) * w.w + (x - w.x0);
    return index >= A.split ? p + (size_t)w.w * w.h : p;
}

__device__ __forceinline__ void adj_add(float* g, uint32_t k, float v) {
    if (v != 0.0f && finitef(v)) atomicAdd(g + k, v);
}

__device__ __forceinline__ float adj_dot(Rgb a, Rgb b) { return a.r * b.r + a.g * b.g + a.b * b.b; }

// Block-level gradient accumulator: a shared copy of the gradient vector, flushed with one global
// atomic per parameter and block.
struct AdjBlock {
    float* g;
    __device__ __forceinline__ void begin(uint32_t n) {
        for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) g[k] = 0.0f;
        __syncthreads();
    }
    __device__ __forceinline__ void end(uint32_t n, float* out) {
        __syncthreads();
        for (uint32_t k = threadIdx.x; k < n; k += blockDim.x)
            if (g[k] != 0.0f) atomicAdd(out + k, g[k]);
    }
};

// The backward wave's camera: the forward's camera rays again, and each slot's radiance still to
// come set to the radiance the forward pass found (left in P.sum).
__global__ void k_adjoint_camera(SceneDev S, WaveDesc w, PathBuffers P, AdjointDev A) {
    float all = 0.0f;
    for (uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x; slot < w.n; slot += gridDim.x * blockDim.x) {
        uint32_t x, y, index;
        wave_slot(w, slot, x, y, index);
        V3 o, d;
        const bool sees = camera_ray(S, c_sobol, x, y, index, o, d);
        P.o[slot] = make_float4(o.x, o.y, o.z, 0.0f);
        P.d[slot] = make_float4(d.x, d.y, d.z, 0.0f);
        // A panoramic camera's sample that sees nothing added nothing to the film: it replays with
        // no throughput and no radiance to come, so it adds no gradient.
        const float w0 = sees ? 1.0f : 0.0f;
        P.thr[slot] = make_float4(w0, w0, w0, 1.0f);
        P.flags[slot] = PF_PRIMARY | (sees ? 0u : PF_NOTHING);
        P.queue[0][slot] = slot;
        float4 L = sees ? P.sum[slot] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        A.rem[slot] = L;
        A.pend[slot] = ADJ_NONE;
        all += absf(L.x) + absf(L.y) + absf(L.z);
    }
    for (int o = 16; o > 0; o >>= 1) all += __shfl_xor_sync(0xffffffffu, all, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(A.residual + 1, all);
    if (blockIdx.x == 0) {
        for (uint32_t k = threadIdx.x; k < 512; k += blockDim.x) P.bins[k] = 0;
        if (threadIdx.x == 0) {
            P.counters[0] = w.n;
            P.counters[1] = 0;
            P.counters[2] = 0;
            P.counters[4] = 0;
            P.counters[5] = 0;
        }
    }
}

// One vertex of the backward wave: the forward's shading (shade_slot) step for step, taking every
// radiance term it adds off the slot's radiance still to come and adding the gradients described
// above. A shadow ray carries its contribution and its material gradient to k_shadow_adjoint.
// The power gradients of the suns an escaping ray sees: each sun's light is proportional to
// its power, so its share of the path's value is <dL, thr L_sun>.
__device__ __noinline__ void adjoint_suns(const LightsDev& L, V3 dir, bool has_pdf, float pdf, const Sel& from, Rgb thr, Rgb dl,
                                          float* g, uint32_t base_light) {
    for (int i = L.n_areas; i < L.n_areas + (int)L.n_suns; ++i) {
        Rgb term;
        if (sun_seen(L, L.lights[i], dir, has_pdf, pdf, from, term)) adj_add(g, base_light + i, adj_dot(dl, thr * term));
    }
}

// crossed plus the sphere lights a ray crosses, each adding <dL, thr L_sphere> to its power's
// gradient.
__device__ __noinline__ Rgb adjoint_spheres(const LightsDev& L, Rgb crossed, V3 ro, V3 rd, float t_nearest, bool has_pdf, float pdf,
                                            const Sel& from, float offset, Rgb thr, Rgb dl, float* g, uint32_t base_light) {
    const int first = L.n_areas + (int)L.n_suns;
    for (int i = first; i < first + (int)L.n_spheres; ++i) {
        Rgb term;
        if (!sphere_crossed(L, L.lights[i], ro, rd, 1.0e-3f, t_nearest, has_pdf, pdf, from, offset, term)) continue;
        crossed = crossed + term;
        adj_add(g, base_light + i, adj_dot(dl, thr * term));
    }
    return crossed;
}

__device__ __forceinline__ void shade_adjoint_slot(const SceneDev& S, const LightsDev& L, const PathBuffers& P, const AdjointDev& A, float* g,
                                                   uint32_t slot, int cur, uint32_t bounce, const WaveDesc& w) {
    float4 o4 = P.o[slot], d4 = P.d[slot], thr4 = P.thr[slot];
    uint32_t flags = P.flags[slot];
    uint4 hit = P.hit[slot];
    V3 ro = v3(o4.x, o4.y, o4.z), rd = v3(d4.x, d4.y, d4.z);
    float offset = o4.w, pdf = d4.w;
    bool has_pdf = (flags & PF_HAS_PDF) != 0, primary = (flags & PF_PRIMARY) != 0;
    Rgb thr = rgb(thr4.x, thr4.y, thr4.z);
    uint32_t x, y, index;
    wave_slot(w, slot, x, y, index);
    const float4 d4p = A.dpath[adj_dpath_index(A, w, x, y, index)];
    const Rgb dl = rgb(d4p.x, d4p.y, d4p.z);
    const float4 r4 = A.rem[slot];
    Rgb rem = rgb(r4.x, r4.y, r4.z);
    const uint32_t base_light = 4 * A.n_materials;
    // The BSDF sample of the last vertex: everything from here on was scaled by its f.
    const uint32_t pm = A.pend[slot];
    if (pm != ADJ_NONE) {
        float4 qa = A.pend_albedo[slot], qr = A.pend_alpha[slot];
        adj_add(g, 4 * pm + 0, dl.r * rem.r * qa.x);
        adj_add(g, 4 * pm + 1, dl.g * rem.g * qa.y);
        adj_add(g, 4 * pm + 2, dl.b * rem.b * qa.z);
        adj_add(g, 4 * pm + 3, dl.r * rem.r * qr.x + dl.g * rem.g * qr.y + dl.b * rem.b * qr.z);
        A.pend[slot] = ADJ_NONE;
    }
    float t_geometry = hit.w ? __uint_as_float(hit.z) : f_inf();
    float t_floor = f_inf();
    if ((S.floor_mode == 1) && rd.z != 0.0f) {
        float t = (S.floor_z - ro.z) / rd.z;
        if (t > 1.0e-3f && t < f_inf()) t_floor = t;
    }
    float t_nearest = rmin(t_geometry, t_floor);
    if ((flags & PF_MEDIUM) && finitef(t_nearest)) {
        const uint32_t medium = P.medium[slot];
        const DevMaterial& mm = S.materials[medium];
        thr = thr * rgb(fexp(-mm.sigma[0] * t_nearest), fexp(-mm.sigma[1] * t_nearest), fexp(-mm.sigma[2] * t_nearest));
        // exp(-sigma t), sigma = -ln(clamp(base, 1e-4, 1)) / absorption: d/d base = t / (base * absorption)
        for (int c = 0; c < 3; ++c) {
            float b = mm.base[c];
            if (b > 1.0e-4f && b < 1.0f) {
                float r = c == 0 ? rem.r : (c == 1 ? rem.g : rem.b);
                float d = c == 0 ? dl.r : (c == 1 ? dl.g : dl.b);
                adj_add(g, 4 * medium + c, d * r * t_nearest / (b * mm.absorption_mm));
            }
        }
    }
    float4 sel4 = P.sel[slot];
    Sel from;
    from.p = v3(sel4.x, sel4.y, sel4.z);
    from.by_flux = !(L.per_point && L.n_entries > 0);
    from.total = 0.0f;
    if (has_pdf && !from.by_flux) from = select_at(L, from.p);
    // crossed_from, light by light, in its order
    Rgb crossed = splat(0.0f);
    for (int i = 0; i < L.n_areas; ++i) {
        const LightDev& l = L.lights[i];
        if (!(has_pdf ? l.glossy : l.camera)) continue;
        float t, cos;
        if (!area_intersect(l, ro, rd, 1.0e-3f, t_nearest, t, cos)) continue;
        float wgt = 1.0f;
        if (has_pdf) {
            float dd = offset + t;
            float light_pdf = pmf_of(L, l.entry, from) * dd * dd / (l.area * cos);
            wgt = power_heuristic(pdf, light_pdf);
        }
        Rgb term = area_radiance(l, cos) * wgt;
        crossed = crossed + term;
        adj_add(g, base_light + i, adj_dot(dl, thr * term));
    }
    if (L.n_spheres) crossed = adjoint_spheres(L, crossed, ro, rd, t_nearest, has_pdf, pdf, from, offset, thr, dl, g, base_light);
    {
        float4 c4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        add_clamped(c4, thr * crossed, bounce >= 2, S.clamp_indirect);
        rem = rgb_sub(rem, rgb(c4.x, c4.y, c4.z));
    }
    bool alive = false;
    do {
        if (t_nearest == f_inf()) {
            if (primary && S.background == 0) {
                Rgb seen = escaped(L, rd, false, 0.0f, from);
                rem = rgb_sub(rem, thr * (S.exterior == 1.0f ? seen : seen * S.exterior));
                if (L.n_suns) adjoint_suns(L, rd, false, 0.0f, from, thr * S.exterior, dl, g, base_light);
            } else if (primary && S.background == 1) {
                rem = rgb_sub(rem, thr * rgb(S.background_color[0], S.background_color[1], S.background_color[2]));
            } else if (!(primary && S.background == 2)) {
                float4 c4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                add_clamped(c4, thr * escaped(L, rd, has_pdf, pdf, from), bounce >= 2, S.clamp_indirect);
                rem = rgb_sub(rem, rgb(c4.x, c4.y, c4.z));
                if (L.n_suns) adjoint_suns(L, rd, has_pdf, pdf, from, thr, dl, g, base_light);
            }
            break;
        }
        V3 s_point, s_hit, s_normal, s_geom;
        bool s_inst = false, s_outside = true;
        const DevInstance* I = nullptr;
        const DevMaterial* mat = nullptr;
        if (t_floor < t_geometry) {
            V3 pp = ro + rd * t_floor;
            V3 point = v3(pp.x, pp.y, S.floor_z);
            V3 nn = v3(0.0f, 0.0f, rd.z < 0.0f ? 1.0f : -1.0f);
            s_point = point; s_hit = point; s_normal = nn; s_geom = nn;
        } else {
            HitInfo h;
            uint4 idx;
            if (!hit_details(S, ro, rd, 1.0e-3f, f_inf(), hit.x, hit.y, __uint_as_float(hit.z), h, I, idx)) break;
            V3 ng = h.geometric, nrm = h.normal;
            if (dot(nrm, ng) < 0.0f) nrm = -nrm;
            if (dot(nrm, rd) >= -1.0e-4f) nrm = ng;
            s_point = terminator_point(S, I, idx, h);
            s_hit = h.point;
            s_normal = nrm;
            s_geom = ng;
            s_inst = true;
            s_outside = h.outside;
            mat = S.materials + I->material;
            if (mat->kind == MATERIAL_EMISSIVE) {
                if (h.front || !(I->flags & 1u)) {
                    const float wgt = has_pdf ? emitter_weight(L, I->emitter, pdf, from, offset + t_geometry, dot(ng, rd)) : 1.0f;
                    float4 c4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                    add_clamped(c4, thr * rgb(mat->emission[0], mat->emission[1], mat->emission[2]) * wgt, bounce >= 2, S.clamp_indirect);
                    rem = rgb_sub(rem, rgb(c4.x, c4.y, c4.z));
                }
                break;
            }
        }
        if (bounce >= S.max_depth) break;
        const uint32_t m = mat ? I->material : 0, side = s_outside ? 0 : 1;
        const Bsdf& b = S.bsdfs[mat ? 2 * m + side : 2 * S.n_materials];
        Frame fr = frame_from_normal(s_normal);
        if (s_inst && I->tangent_on) {
            V3 cands[2] = {cross(ld3(I->tan_axis), s_point - ld3(I->tan_centre)), ld3(I->tan_x)};
            for (int k = 0; k < 2; ++k) {
                V3 t = cands[k] - s_normal * dot(s_normal, cands[k]);
                if (len2(t) > 1.0e-12f) {
                    V3 xx = normalize(t);
                    fr.x = xx; fr.y = cross(s_normal, xx); fr.z = s_normal;
                    break;
                }
            }
        }
        V3 wo = to_local(fr, -rd);
        V3 ng = s_geom;
        V3 origin = offset_origin(s_point, ng);
        uint32_t dims = bounce_dim(bounce);
        uint64_t key = sample_key(S, x, y, index);
        Sel selection = select_at(L, s_point);
        LightSample ls;
        if (sample_light(L, selection, sample1(c_sobol, key, index, dims + OFF_LIGHT_SELECT), sample1(c_sobol, key, index, dims + OFF_LIGHT),
                         sample1(c_sobol, key, index, dims + OFF_LIGHT + 1), ls)) {
            V3 wi = to_local(fr, ls.wi);
            const LobesSel lobes = ls.glossy ? LOBES_ALL : LOBES_DIFFUSE;
            Rgb f = bsdf_eval(S.energy, b, wo, wi, lobes);
            if (peak(f) > 0.0f) {
                V3 from_p = wi.z < 0.0f ? offset_origin(s_hit, -ng) : origin;
                float weight = (ls.delta || !ls.glossy) ? 1.0f : power_heuristic(ls.pdf, bsdf_pdf(S.energy, b, wo, wi));
                float kscale = absf(wi.z) * weight / ls.pdf;
                Rgb c = thr * f * ls.radiance * kscale;
                bool finite_c = finitef(c.r) && finitef(c.g) && finitef(c.b);
                float clamp_scale = 1.0f;
                if (finite_c && bounce >= 1 && S.clamp_indirect > 0.0f) {
                    float p = rmax(rmax(c.r, c.g), c.b);
                    if (p > S.clamp_indirect) {
                        clamp_scale = S.clamp_indirect / p;
                        c = c * clamp_scale;
                    }
                }
                // The material gradient of this estimate, should it count: <dL, K df>, c = K f.
                float4 mg = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                if (mat && finite_c) {
                    Rgb K = thr * ls.radiance * (kscale * clamp_scale);
                    const uint32_t k = 2 * m + side;
                    Rgb fa = rgb_sub(bsdf_eval(S.energy, A.albedo_plus[k], wo, wi, lobes), bsdf_eval(S.energy, A.albedo_minus[k], wo, wi, lobes)) *
                             A.inv_2h_albedo;
                    Rgb fr2 = rgb_sub(bsdf_eval(S.energy, A.alpha_plus[k], wo, wi, lobes), bsdf_eval(S.energy, A.alpha_minus[k], wo, wi, lobes)) *
                              A.inv_2h_alpha;
                    mg = make_float4(dl.r * K.r * fa.r, dl.g * K.g * fa.g, dl.b * K.b * fa.b,
                                     dl.r * K.r * fr2.r + dl.g * K.g * fr2.g + dl.b * K.b * fr2.b);
                }
                if (!ls.shadow) {
                    if (finite_c) {
                        rem = rgb_sub(rem, c);
                        if (ls.light >= 0) adj_add(g, base_light + (uint32_t)ls.light, adj_dot(dl, c));
                        if (mat) {
                            adj_add(g, 4 * m + 0, mg.x);
                            adj_add(g, 4 * m + 1, mg.y);
                            adj_add(g, 4 * m + 2, mg.z);
                            adj_add(g, 4 * m + 3, mg.w);
                        }
                    }
                } else {
                    float tmax = finitef(ls.distance) ? ls.distance * (1.0f - 1.0e-4f) : f_inf();
                    bool floor_blocks = false;
                    if (S.floor_mode == 1 && ls.wi.z != 0.0f) {
                        float t = (S.floor_z - from_p.z) / ls.wi.z;
                        floor_blocks = t > 1.0e-3f && t < tmax;
                    }
                    if (finite_c && !floor_blocks) {
                        uint32_t k = atomicAdd(&P.counters[2], 1u);
                        P.sh_o[k] = make_float4(from_p.x, from_p.y, from_p.z, tmax);
                        P.sh_d[k] = make_float4(ls.wi.x, ls.wi.y, ls.wi.z, 0.0f);
                        P.sh_c[k] = make_float4(c.r, c.g, c.b, __uint_as_float(slot));
                        A.sh_grad[k] = mg;
                        A.sh_ids[k] = (mat ? m + 1 : 0u) | ((uint32_t)(ls.light + 1) << 16);
                    }
                }
            }
        }
        BsdfSample bs;
        if (!bsdf_sample(S.energy, b, wo, sample1(c_sobol, key, index, dims + OFF_BSDF), sample1(c_sobol, key, index, dims + OFF_BSDF + 1), bs))
            break;
        bool transmitted = bs.wi.z < 0.0f;
        V3 wi = bs.straight ? rd : normalize(to_world(fr, bs.wi));
        if (transmitted) {
            if (dot(wi, ng) >= 0.0f) break;
        } else if (dot(wi, ng) <= 0.0f) {
            break;
        }
        thr = thr * bs.weight;
        if (bounce >= 2) {
            float survive = rclamp(peak(thr), 0.05f, 1.0f);
            if (sample1(c_sobol, key, index, dims + OFF_ROULETTE) >= survive) break;
            thr = thr / survive;
        }
        float pk = peak(thr);
        if (!(pk > 0.0f && finitef(pk))) break;
        // Everything after this vertex is scaled by f(wo, wi) / pdf: d/d theta = rem * df / f,
        // applied when the next vertex knows rem.
        if (mat && !bs.straight) {
            const uint32_t k = 2 * m + side;
            Rgb f = bsdf_eval(S.energy, b, wo, bs.wi, LOBES_ALL);
            Rgb fa = rgb_sub(bsdf_eval(S.energy, A.albedo_plus[k], wo, bs.wi, LOBES_ALL), bsdf_eval(S.energy, A.albedo_minus[k], wo, bs.wi, LOBES_ALL)) *
                     A.inv_2h_albedo;
            Rgb fr2 = rgb_sub(bsdf_eval(S.energy, A.alpha_plus[k], wo, bs.wi, LOBES_ALL), bsdf_eval(S.energy, A.alpha_minus[k], wo, bs.wi, LOBES_ALL)) *
                      A.inv_2h_alpha;
            A.pend[slot] = m;
            A.pend_albedo[slot] = make_float4(f.r > 0.0f ? fa.r / f.r : 0.0f, f.g > 0.0f ? fa.g / f.g : 0.0f, f.b > 0.0f ? fa.b / f.b : 0.0f, 0.0f);
            A.pend_alpha[slot] = make_float4(f.r > 0.0f ? fr2.r / f.r : 0.0f, f.g > 0.0f ? fr2.g / f.g : 0.0f, f.b > 0.0f ? fr2.b / f.b : 0.0f, 0.0f);
        }
        V3 next_origin = transmitted ? offset_origin(s_hit, -ng) : origin;
        if (bs.straight) {
            offset += dot(next_origin - ro, rd);
        } else {
            flags |= PF_HAS_PDF;
            flags &= ~PF_PRIMARY;
            pdf = bs.pdf;
            P.sel[slot] = make_float4(s_point.x, s_point.y, s_point.z, 0.0f);
            offset = 0.0f;
            if (transmitted) {
                if (s_outside && mat && mat->has_medium) {
                    flags |= PF_MEDIUM;
                    P.medium[slot] = I->material;
                } else {
                    flags &= ~PF_MEDIUM;
                }
            }
        }
        P.o[slot] = make_float4(next_origin.x, next_origin.y, next_origin.z, offset);
        P.d[slot] = make_float4(wi.x, wi.y, wi.z, pdf);
        P.flags[slot] = flags;
        alive = true;
    } while (false);
    P.thr[slot] = make_float4(thr.r, thr.g, thr.b, thr4.w);
    A.rem[slot] = make_float4(rem.r, rem.g, rem.b, 0.0f);
    if (alive) {
        uint32_t k = atomicAdd(&P.counters[cur ^ 1], 1u);
        P.queue[cur ^ 1][k] = slot;
    }
}

// Eight blocks per SM (64 registers, with spills) rather than the compiler's 168 registers: as for
// k_shade, more warps hide the scattered loads (512^2 adjoint iteration 51.4 -> 48.9 ms).
__global__ void __launch_bounds__(128, RTG_SHADE_MIN_BLOCKS) k_shade_adjoint(SceneDev S, const LightsDev* __restrict__ Lg, PathBuffers P, int cur, uint32_t bounce,
                                                       WaveDesc w, AdjointDev A) {
    __shared__ float s_grad[MAX_ADJOINT_PARAMS];
    AdjBlock blk{s_grad};
    const uint32_t n_params = 4 * A.n_materials + A.n_lights;
    blk.begin(n_params);
    uint32_t n = *(volatile uint32_t*)&P.counters[cur];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        shade_adjoint_slot(S, *Lg, P, A, s_grad, P.sorted[i], cur, bounce, w);
    blk.end(n_params, A.grads);
}

// Shadow rays of the backward wave: an unblocked one takes its contribution off its path's
// radiance still to come and adds its light's and its material's gradients. Persistent warps
// with lane refill, as k_shadow.
__device__ __forceinline__ void adjoint_unblocked(const PathBuffers& P, const AdjointDev& A, const WaveDesc& w, float* g, uint32_t i) {
    const float4 c = P.sh_c[i];
    const uint32_t slot = __float_as_uint(c.w);
    float4 r = A.rem[slot];
    r.x = r.x - c.x; r.y = r.y - c.y; r.z = r.z - c.z;
    A.rem[slot] = r;
    uint32_t x, y, index;
    wave_slot(w, slot, x, y, index);
    const float4 d4p = A.dpath[adj_dpath_index(A, w, x, y, index)];
    const uint32_t ids = A.sh_ids[i], m1 = ids & 0xffffu, a1 = ids >> 16;
    if (a1) adj_add(g, 4 * A.n_materials + a1 - 1, d4p.x * c.x + d4p.y * c.y + d4p.z * c.z);
    if (m1) {
        const float4 mg = A.sh_grad[i];
        adj_add(g, 4 * (m1 - 1) + 0, mg.x);
        adj_add(g, 4 * (m1 - 1) + 1, mg.y);
        adj_add(g, 4 * (m1 - 1) + 2, mg.z);
        adj_add(g, 4 * (m1 - 1) + 3, mg.w);
    }
}

__global__ void __launch_bounds__(TRACE_THREADS) k_shadow_adjoint(SceneDev S, PathBuffers P, WaveDesc w, AdjointDev A) {
    __shared__ uint64_t s_stack[SHORT_STACK * TRACE_THREADS];
    __shared__ float s_grad[MAX_ADJOINT_PARAMS];
    uint64_t deep[STACK_CAP - SHORT_STACK];
    SplitStack stack{s_stack + threadIdx.x, deep, TRACE_THREADS};
    AdjBlock blk{s_grad};
    const uint32_t n_params = 4 * A.n_materials + A.n_lights;
    blk.begin(n_params);
    const uint32_t n = *(volatile uint32_t*)&P.counters[2];
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t err = 0, ray = 0;
    bool busy = false, drained = false;
    Trav T;
    for (;;) {
        if (!drained) {
            const uint32_t idle = __ballot_sync(0xffffffffu, !busy);
            // k_shadow's refill threshold (RTG_SHADOW_REFILL_MIN idle lanes, or all of them)
            if (idle && (RTG_SHADOW_REFILL_MIN <= 1 || __popc(idle) >= RTG_SHADOW_REFILL_MIN || idle == 0xffffffffu)) {
                const int leader = __ffs((int)idle) - 1;
                uint32_t base = 0;
                if ((int)lane == leader) base = atomicAdd(&P.counters[5], (uint32_t)__popc(idle));
                base = __shfl_sync(0xffffffffu, base, leader);
                if (base + (uint32_t)__popc(idle) >= n) drained = true;
                const uint32_t i = base + (uint32_t)__popc(idle & ((1u << lane) - 1u));
                if (!busy && i < n) {
                    ray = i;
                    const float4 o = P.sh_o[i], d = P.sh_d[i];
                    busy = trav_init(S, T, v3(o.x, o.y, o.z), v3(d.x, d.y, d.z), 1.0e-3f, o.w, false);
                    if (!busy) adjoint_unblocked(P, A, w, s_grad, i);
                }
            }
        }
        if (!__any_sync(0xffffffffu, busy)) {
            if (drained) break;
            continue;
        }
        if (busy) {
            bool blocked = false;
            if (trav_step<true>(S, T, stack, &err, blocked)) {
                busy = false;
                if (!blocked) adjoint_unblocked(P, A, w, s_grad, ray);
            }
        }
    }
    blk.end(n_params, A.grads);
    if (err) atomicOr(&P.counters[3], err);
}

// Sum over the paths with a loss derivative of |radiance left| after the backward wave.
__global__ void k_adjoint_residual(WaveDesc w, PathBuffers P, AdjointDev A) {
    float left = 0.0f;
    for (uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x; slot < w.n; slot += gridDim.x * blockDim.x) {
        float4 r = A.rem[slot];
        left += absf(r.x) + absf(r.y) + absf(r.z);
    }
    for (int o = 16; o > 0; o >>= 1) left += __shfl_xor_sync(0xffffffffu, left, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(A.residual, left);
}

// The loss L = mean over the film's pixels and channels of (I - T)^2, I = rgb / weight (all the
// call's samples), summed in double, and the per-pixel loss derivatives the backward wave uses.
// An L2 gradient whose residual I - T and derivative dI/dtheta come from the same paths is biased
// (their noise is correlated). So the call's `count` samples of each pixel (slots s * npix + p of
// the wave, s < count) are split at h = count / 2 into halves A and B with means I_A, I_B, and
//   dL/dtheta = 1/2 [ sum_p 2 (I_B - T) / (3 npix) dI_A/dtheta + sum_p 2 (I_A - T) / (3 npix) dI_B/dtheta ],
// an unbiased estimate: a path of half A gets dpath[p] = (I_B - T) / (3 npix h), one of half B
// dpath[npix + p] = (I_A - T) / (3 npix (count - h)). With one sample the halves coincide (the
// correlated estimate 2 (I - T) / (3 npix)).
__global__ void k_adjoint_delta(FilmDev F, const float* __restrict__ target, float4* dpath, double* loss, PathBuffers P, uint32_t count) {
    const uint32_t npix = F.w * F.h;
    const uint32_t h = count / 2;  // count 1: one estimate from all samples (the correlated one)
    double local = 0.0;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += gridDim.x * blockDim.x) {
        float wt = F.weight[p];
        float inv = wt > 0.0f ? 1.0f / wt : 0.0f;
        float sa[3] = {0.0f, 0.0f, 0.0f}, sb[3] = {0.0f, 0.0f, 0.0f};
        for (uint32_t k = 0; k < count; ++k) {
            float4 c = P.sum[(size_t)k * npix + p];
            float* acc = k < h ? sa : sb;
            acc[0] = acc[0] + c.x; acc[1] = acc[1] + c.y; acc[2] = acc[2] + c.z;
        }
        float da[3], db[3];
        for (int c = 0; c < 3; ++c) {
            float T = target[3 * p + c];
            float e = F.rgb[3 * p + c] * inv - T;
            local += (double)e * (double)e;
            if (h == 0) {
                da[c] = db[c] = wt > 0.0f ? 2.0f * e / (3.0f * (float)npix * wt) : 0.0f;
            } else {
                float ia = sa[c] / (float)h, ib = sb[c] / (float)(count - h);
                da[c] = (ib - T) / (3.0f * (float)npix * (float)h);
                db[c] = (ia - T) / (3.0f * (float)npix * (float)(count - h));
            }
        }
        dpath[p] = make_float4(da[0], da[1], da[2], 0.0f);
        dpath[npix + p] = make_float4(db[0], db[1], db[2], 0.0f);
    }
    for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, local / (3.0 * (double)npix));
}

}  // namespace rtg
