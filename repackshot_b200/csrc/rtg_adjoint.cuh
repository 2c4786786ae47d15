// The adjoint of the path tracer: gradients of an image loss with respect to every material's base
// colour and GGX alpha and every area light's power, by path replay backpropagation (Vicini,
// Speierer and Jakob, "Path Replay Backpropagation", SIGGRAPH 2021). Included by rtg_kernels.cu,
// whose sampler table and helpers it shares.
//
// A forward wave renders every path of the call and leaves each path's radiance L in its slot.
// k_adjoint_delta turns the film and the target image into the loss and, per pixel, the loss's
// derivative with respect to one path's radiance. k_adjoint_replay then runs every path again
// from its pixel and sample index (the sampler makes it the same path), carrying
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

constexpr int MAX_ADJOINT_PARAMS = 4 * 64 + MAX_AREAS;


__device__ __forceinline__ Rgb rgb_sub(Rgb a, Rgb b) { return rgb(a.r - b.r, a.g - b.g, a.b - b.b); }

__device__ __forceinline__ void adj_add(float* g, uint32_t k, float v) {
    if (v != 0.0f && finitef(v)) atomicAdd(g + k, v);
}

// Material m's BSDF gradient at (wo, wi) for a radiance `scale` that is multiplied by f there:
// albedo channel c gains dL_c scale_c df_c; alpha gains the sum over channels.
__device__ __forceinline__ void adj_bsdf(const AdjointDev& A, float* g, uint32_t m, uint32_t side, V3 wo, V3 wi, LobesSel lobes, Rgb dl,
                                         Rgb scale, const EnergyTables& E) {
    const uint32_t k = 2 * m + side;
    Rgb fa = rgb_sub(bsdf_eval(E, A.albedo_plus[k], wo, wi, lobes), bsdf_eval(E, A.albedo_minus[k], wo, wi, lobes)) * A.inv_2h_albedo;
    Rgb fr = rgb_sub(bsdf_eval(E, A.alpha_plus[k], wo, wi, lobes), bsdf_eval(E, A.alpha_minus[k], wo, wi, lobes)) * A.inv_2h_alpha;
    adj_add(g, 4 * m + 0, dl.r * scale.r * fa.r);
    adj_add(g, 4 * m + 1, dl.g * scale.g * fa.g);
    adj_add(g, 4 * m + 2, dl.b * scale.b * fa.b);
    adj_add(g, 4 * m + 3, dl.r * scale.r * fr.r + dl.g * scale.g * fr.g + dl.b * scale.b * fr.b);
}

__device__ __forceinline__ float adj_dot(Rgb a, Rgb b) { return a.r * b.r + a.g * b.g + a.b * b.b; }

// Replays every path of the wave (one thread each) and accumulates the gradients: per block in
// shared memory, then one global atomic per parameter and block.
__global__ void __launch_bounds__(TRACE_THREADS) k_adjoint_replay(SceneDev S, const LightsDev* __restrict__ Lg, PathBuffers P, WaveDesc w,
                                                                  AdjointDev A) {
    __shared__ uint64_t s_stack[SHORT_STACK * TRACE_THREADS];
    __shared__ float s_grad[MAX_ADJOINT_PARAMS];
    uint64_t deep[STACK_CAP - SHORT_STACK];
    SplitStack stack{s_stack + threadIdx.x, deep, TRACE_THREADS};
    const uint32_t n_params = 4 * A.n_materials + A.n_areas;
    for (uint32_t k = threadIdx.x; k < n_params; k += blockDim.x) s_grad[k] = 0.0f;
    __syncthreads();
    const LightsDev& L = *Lg;
    const uint32_t base_light = 4 * A.n_materials;
    uint32_t err = 0;
    float res_rem = 0.0f, res_all = 0.0f;
    for (uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x; slot < w.n; slot += gridDim.x * blockDim.x) {
        uint32_t x, y, index;
        wave_slot(w, slot, x, y, index);
        const float4 d4p = A.dpath[(size_t)(y - w.y0) * w.w + (x - w.x0)];
        const Rgb dl = rgb(d4p.x, d4p.y, d4p.z);
        const float4 L4 = P.sum[slot];
        Rgb rem = rgb(L4.x, L4.y, L4.z);
        if (dl.r == 0.0f && dl.g == 0.0f && dl.b == 0.0f) continue;
        res_all += absf(rem.r) + absf(rem.g) + absf(rem.b);
        // The path again, step for step as the forward kernels take it (k_camera, k_extend,
        // k_shade, k_shadow); every radiance term the forward adds is taken off `rem`.
        V3 ro, rd;
        camera_ray(S, c_sobol, x, y, index, ro, rd);
        float offset = 0.0f, pdf = 0.0f;
        uint32_t flags = PF_PRIMARY, medium = 0;
        Rgb thr = splat(1.0f);
        V3 selp = v3(0.0f, 0.0f, 0.0f);
        const uint64_t key = pixel_key(S.seed, x, y);
        for (uint32_t bounce = 0;; ++bounce) {
            const bool has_pdf = (flags & PF_HAS_PDF) != 0, primary = (flags & PF_PRIMARY) != 0;
            TraceResult hit;
            const bool got = traverse<false>(S, ro, rd, 1.0e-3f, f_inf(), primary, hit, &err, stack);
            const float t_geometry = got ? hit.t : f_inf();
            float t_floor = f_inf();
            if ((S.floor_mode == 1) && rd.z != 0.0f) {
                float t = (S.floor_z - ro.z) / rd.z;
                if (t > 1.0e-3f && t < f_inf()) t_floor = t;
            }
            const float t_nearest = rmin(t_geometry, t_floor);
            if ((flags & PF_MEDIUM) && finitef(t_nearest)) {
                const DevMaterial& mm = S.materials[medium];
                thr = thr * rgb(fexp(-mm.sigma[0] * t_nearest), fexp(-mm.sigma[1] * t_nearest), fexp(-mm.sigma[2] * t_nearest));
                // exp(-sigma t), sigma = -ln(clamp(base, 1e-4, 1)) / absorption: d/d base = t / (base * absorption)
                for (int c = 0; c < 3; ++c) {
                    float b = mm.base[c];
                    if (b > 1.0e-4f && b < 1.0f) {
                        float r = c == 0 ? rem.r : (c == 1 ? rem.g : rem.b);
                        float d = c == 0 ? dl.r : (c == 1 ? dl.g : dl.b);
                        adj_add(s_grad, 4 * medium + c, d * r * t_nearest / (b * mm.absorption_mm));
                    }
                }
            }
            Sel from;
            from.p = selp;
            from.by_flux = !(L.per_point && L.n_entries > 0);
            from.total = 0.0f;
            if (has_pdf && !from.by_flux) from = select_at(L, from.p);
            // crossed_from, light by light, in its order
            Rgb crossed = splat(0.0f);
            for (int i = 0; i < L.n_areas; ++i) {
                const AreaLightDev& l = L.areas[i];
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
                adj_add(s_grad, base_light + i, adj_dot(dl, thr * term));
            }
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
                    } else if (primary && S.background == 1) {
                        rem = rgb_sub(rem, thr * rgb(S.background_color[0], S.background_color[1], S.background_color[2]));
                    } else if (!(primary && S.background == 2)) {
                        float4 c4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                        add_clamped(c4, thr * escaped(L, rd, has_pdf, pdf, from), bounce >= 2, S.clamp_indirect);
                        rem = rgb_sub(rem, rgb(c4.x, c4.y, c4.z));
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
                    if (!hit_details(S, ro, rd, 1.0e-3f, f_inf(), hit.inst, hit.tri, h, I, idx)) break;
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
                            float4 c4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                            add_clamped(c4, thr * rgb(mat->emission[0], mat->emission[1], mat->emission[2]) * 1.0f, bounce >= 2,
                                        S.clamp_indirect);
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
                // next-event estimation, its shadow ray traced here
                Sel selection = select_at(L, s_point);
                LightSample ls;
                if (sample_light(L, selection, sample1(c_sobol, key, index, dims + OFF_LIGHT_SELECT), sample1(c_sobol, key, index, dims + OFF_LIGHT),
                                 sample1(c_sobol, key, index, dims + OFF_LIGHT + 1), ls)) {
                    V3 wi = to_local(fr, ls.wi);
                    const LobesSel lobes = ls.glossy ? LOBES_ALL : LOBES_DIFFUSE;
                    Rgb f = bsdf_eval(S.energy, b, wo, wi, lobes);
                    if (peak(f) > 0.0f) {
                        V3 from_p = wi.z < 0.0f ? offset_origin(s_hit, -ng) : origin;
                        float weight = !ls.glossy ? 1.0f : power_heuristic(ls.pdf, bsdf_pdf(S.energy, b, wo, wi));
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
                        bool adds = false;
                        if (!ls.shadow) {
                            adds = finite_c;
                        } else {
                            float tmax = finitef(ls.distance) ? ls.distance * (1.0f - 1.0e-4f) : f_inf();
                            bool floor_blocks = false;
                            if (S.floor_mode == 1 && ls.wi.z != 0.0f) {
                                float t = (S.floor_z - from_p.z) / ls.wi.z;
                                floor_blocks = t > 1.0e-3f && t < tmax;
                            }
                            if (finite_c && !floor_blocks) {
                                TraceResult sh;
                                adds = !traverse<true>(S, from_p, ls.wi, 1.0e-3f, tmax, false, sh, &err, stack);
                            }
                        }
                        if (adds) {
                            rem = rgb_sub(rem, c);
                            if (ls.area >= 0) adj_add(s_grad, base_light + (uint32_t)ls.area, adj_dot(dl, c));
                            if (mat) adj_bsdf(A, s_grad, m, side, wo, wi, lobes, dl, thr * ls.radiance * (kscale * clamp_scale), S.energy);
                        }
                    }
                }
                // the next direction
                BsdfSample bs;
                if (!bsdf_sample(S.energy, b, wo, sample1(c_sobol, key, index, dims + OFF_BSDF), sample1(c_sobol, key, index, dims + OFF_BSDF + 1),
                                 bs))
                    break;
                bool transmitted = bs.wi.z < 0.0f;
                V3 wi = bs.straight ? rd : normalize(to_world(fr, bs.wi));
                if (transmitted) {
                    if (dot(wi, ng) >= 0.0f) break;
                } else if (dot(wi, ng) <= 0.0f) {
                    break;
                }
                // Everything after this vertex is scaled by f(wo, wi) / pdf: d/d theta = rem * df / f.
                if (mat && !bs.straight) {
                    Rgb f = bsdf_eval(S.energy, b, wo, bs.wi, LOBES_ALL);
                    Rgb q = rgb(f.r > 0.0f ? rem.r / f.r : 0.0f, f.g > 0.0f ? rem.g / f.g : 0.0f, f.b > 0.0f ? rem.b / f.b : 0.0f);
                    adj_bsdf(A, s_grad, m, side, wo, bs.wi, LOBES_ALL, dl, q, S.energy);
                }
                thr = thr * bs.weight;
                if (bounce >= 2) {
                    float survive = rclamp(peak(thr), 0.05f, 1.0f);
                    if (sample1(c_sobol, key, index, dims + OFF_ROULETTE) >= survive) break;
                    thr = thr / survive;
                }
                float pk = peak(thr);
                if (!(pk > 0.0f && finitef(pk))) break;
                V3 next_origin = transmitted ? offset_origin(s_hit, -ng) : origin;
                if (bs.straight) {
                    offset += dot(next_origin - ro, rd);
                } else {
                    flags |= PF_HAS_PDF;
                    flags &= ~PF_PRIMARY;
                    pdf = bs.pdf;
                    selp = s_point;
                    offset = 0.0f;
                    if (transmitted) {
                        if (s_outside && mat && mat->has_medium) {
                            flags |= PF_MEDIUM;
                            medium = I->material;
                        } else {
                            flags &= ~PF_MEDIUM;
                        }
                    }
                }
                ro = next_origin;
                rd = wi;
                alive = true;
            } while (false);
            if (!alive) break;
        }
        res_rem += absf(rem.r) + absf(rem.g) + absf(rem.b);
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < n_params; k += blockDim.x)
        if (s_grad[k] != 0.0f) atomicAdd(A.grads + k, s_grad[k]);
    for (int o = 16; o > 0; o >>= 1) {
        res_rem += __shfl_xor_sync(0xffffffffu, res_rem, o);
        res_all += __shfl_xor_sync(0xffffffffu, res_all, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(A.residual, res_rem);
        atomicAdd(A.residual + 1, res_all);
    }
    if (err) atomicOr(&P.counters[3], err);
}

// The loss L = mean over the film's pixels and channels of (I - T)^2, I = rgb / weight, and per
// pixel dL/d(one path's radiance) = 2 (I - T) / (3 npix weight). Sums the loss in double.
__global__ void k_adjoint_delta(FilmDev F, const float* __restrict__ target, float4* dpath, double* loss) {
    const uint32_t npix = F.w * F.h;
    double local = 0.0;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += gridDim.x * blockDim.x) {
        float wt = F.weight[p];
        float inv = wt > 0.0f ? 1.0f / wt : 0.0f;
        float d[3];
        for (int c = 0; c < 3; ++c) {
            float I = F.rgb[3 * p + c] * inv;
            float e = I - target[3 * p + c];
            local += (double)e * (double)e;
            d[c] = wt > 0.0f ? 2.0f * e / (3.0f * (float)npix * wt) : 0.0f;
        }
        dpath[p] = make_float4(d[0], d[1], d[2], 0.0f);
    }
    for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, local / (3.0 * (double)npix));
}

}  // namespace rtg
