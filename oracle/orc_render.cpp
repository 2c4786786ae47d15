// ORACLE (test infrastructure only). The path tracer and the tile renderer restated from
// engine/crates/rt-core/src/integrator/mod.rs:237-1891 and render.rs:79-497, plus the C entry
// points the tests and the CPU baseline call through ctypes. Nothing in the product links this.
#include <atomic>
#include <cstdio>
#include <memory>
#include <mutex>
#include <thread>

#include "orc_adaptive.h"
#include "orc_scene.h"

namespace orc {

struct PathStats;

struct Prepared {  // integrator/mod.rs:237
    Lights lights;
    uint32_t background = 0;  // 0 environment, 1 colour, 2 transparent, 3 backplate
    Rgb background_color;
    // The background image fitted to the frame (integrator/mod.rs:187).
    const Image* plate = nullptr;
    uint32_t plate_fit = 0;  // 0 fill, 1 fit, 2 stretch
    float plate_rect[4] = {0.0f, 0.0f, 1.0f, 1.0f};
    float frame_aspect = 1.0f, image_aspect = 1.0f;
    // Per instance: shadow rays may pass it (a cut-out or a thin wall).
    std::vector<uint8_t> passable;
    bool any_passable = false;
    uint32_t floor_mode = 0;
    float floor_z = 0;
    Bsdf floor_bsdf;
    uint32_t max_depth = 8;
    float clamp_indirect = 0;
    Material fallback;
    std::vector<bool> has_medium;
    std::vector<Rgb> media;  // per material: absorption per mm
    struct Axes { bool on = false; Vec3 centre, axis, x_axis; };
    std::vector<Axes> tangent_axes;

    static Prepared make(const Scene& s);
    float floor_t(const Ray& ray, bool camera_ray) const {
        bool present = floor_mode == 1 || (floor_mode == 2 && camera_ray);
        if (!present || ray.dir.z == 0.0f) return F_INF;
        float t = (floor_z - ray.origin.z) / ray.dir.z;
        return (t > ray.t_min && t < ray.t_max) ? t : F_INF;
    }
    const Material& material(const Scene& s, uint32_t inst) const {
        if (inst < s.geometry.instances.size()) {
            uint32_t id = s.geometry.instances[inst].material_id;
            if (id < s.materials.size()) return s.materials[id];
        }
        return fallback;
    }
    Frame frame(bool has_inst, uint32_t inst, Vec3 point, Vec3 n) const {  // integrator/mod.rs:833
        if (has_inst && inst < tangent_axes.size() && tangent_axes[inst].on) {
            const Axes& a = tangent_axes[inst];
            Vec3 cands[2] = {cross(a.axis, point - a.centre), a.x_axis};
            for (Vec3 t : cands) {
                t = t - n * dot(n, t);
                if (length_squared(t) > 1.0e-12f) {
                    Vec3 x = normalize(t);
                    Frame f;
                    f.x = x;
                    f.y = cross(n, x);
                    f.z = n;
                    return f;
                }
            }
        }
        return Frame::from_normal(n);
    }
    // Backplate::lookup (integrator/mod.rs:201): the image at screen position (su, sv), false
    // outside a fitted image.
    bool lookup(float su, float sv, Rgb& out) const {
        float u = (su - plate_rect[0]) / (plate_rect[2] - plate_rect[0]);
        float v = (sv - plate_rect[1]) / (plate_rect[3] - plate_rect[1]);
        if (plate_fit != 2) {
            bool fit = plate_fit == 1;
            float k = frame_aspect / image_aspect;
            if (image_aspect > frame_aspect) {
                if (fit) v = 0.5f + (v - 0.5f) * (1.0f / k);
                else u = 0.5f + (u - 0.5f) * k;
            } else if (fit) {
                u = 0.5f + (u - 0.5f) * k;
            } else {
                v = 0.5f + (v - 0.5f) * (image_aspect / frame_aspect);
            }
        }
        if (plate_fit == 1 && !(u >= 0.0f && u <= 1.0f && v >= 0.0f && v <= 1.0f)) return false;
        out = plate->bilinear(rclamp(u, 0.0f, 1.0f), rclamp(v, 0.0f, 1.0f), false);
        return true;
    }
    Rgb backdrop(float su, float sv) const {  // integrator/mod.rs:867
        Rgb c;
        if (plate && background == 3 && lookup(su, sv, c)) return c;
        return background_color;
    }
    // What a straight ray through the surface keeps, and where it goes on from: a cut-out lets
    // 1 - opacity through, a thin wall its straight transmittance (integrator/mod.rs:581).
    Rgb straight_through(const Scene& s, const Ray& r, uint32_t inst, const Hit& d, Vec3& origin) const {
        const Material& m = material(s, inst);
        float cos = dot(d.geometric_normal, r.dir);
        float opacity = rclamp(m.opacity, 0.0f, 1.0f);
        origin = offset_origin(d.point, -d.geometric_normal);
        return Bsdf::surface(m, true).straight_transmittance(cos) * opacity + Rgb::splat(1.0f - opacity);
    }
    // Prepared::shadow (integrator/mod.rs:681) with Prepared::walk (integrator/mod.rs:629): false
    // when the geometry or the visible floor blocks the ray, else what passes.
    bool shadow(const Scene& s, const Ray& ray, Rgb& pass, PathStats& st) const;
    void add(Rgb& sum, Rgb c, bool indirect) const {  // integrator/mod.rs:855
        if (!(finite(c.r) && finite(c.g) && finite(c.b))) return;
        float p = rmax(rmax(c.r, c.g), c.b);
        if (indirect && clamp_indirect > 0.0f && p > clamp_indirect) sum = sum + c * (clamp_indirect / p);
        else sum = sum + c;
    }
};

Prepared Prepared::make(const Scene& s) {
    Prepared p;
    const Environment& env = s.environment;
    if (env.backplate_map != NO_BITMAP && env.backplate_map < s.bitmaps.size()) {
        p.plate = &s.bitmaps[env.backplate_map];
        uint32_t w = s.render.width ? s.render.width : 1, h = s.render.height ? s.render.height : 1;
        const float* r = env.backplate_rect;
        if (r[2] > r[0] && r[3] > r[1]) for (int k = 0; k < 4; ++k) p.plate_rect[k] = r[k];
        p.plate_fit = env.backplate_fit;
        p.frame_aspect = ((p.plate_rect[2] - p.plate_rect[0]) * (float)w) / ((p.plate_rect[3] - p.plate_rect[1]) * (float)h);
        p.image_aspect = (float)p.plate->width / (float)p.plate->height;
    }
    p.background = env.background_mode == 1 ? 1 : env.background_mode == 2 ? 2 : env.background_mode == 3 ? (p.plate ? 3 : 1) : 0;
    p.background_color = Rgb(rmax(env.background_color.r, 0.0f), rmax(env.background_color.g, 0.0f), rmax(env.background_color.b, 0.0f));
    p.floor_mode = s.floor.mode;
    p.floor_z = s.floor.z;
    p.floor_bsdf = Bsdf::lambert(s.floor.color);
    p.max_depth = s.render.depth();
    p.clamp_indirect = s.render.clamp_indirect;
    for (const Material& m : s.materials) {
        // medium_of (integrator/mod.rs:298)
        bool clear = m.transmission > 0.0f && m.metallic < 1.0f && (m.flags & MATERIAL_FLAG_THIN) == 0;
        bool on = false;
        Rgb sigma;
        if (clear && m.absorption_mm > 0.0f && !m.is_emissive()) {
            auto f = [&](float c) { return -fln(rclamp(c, 1.0e-4f, 1.0f)) / m.absorption_mm; };
            sigma = Rgb(f(m.base_color.r), f(m.base_color.g), f(m.base_color.b));
            on = sigma.r > 0.0f || sigma.g > 0.0f || sigma.b > 0.0f;
        }
        p.has_medium.push_back(on);
        p.media.push_back(sigma);
    }
    const Geometry& g = s.geometry;
    for (size_t i = 0; i < g.instances.size(); ++i) {  // integrator/mod.rs:371
        const Material& m = p.material(s, (uint32_t)i);
        bool thin = (m.flags & MATERIAL_FLAG_THIN) != 0;
        bool pass = g.instances[i].material_id < s.materials.size() && !m.is_emissive() &&
                    (m.opacity < 1.0f || (thin && m.transmission > 0.0f && (m.metallic < 1.0f || m.kind == MATERIAL_GLASS)));
        p.passable.push_back(pass ? 1 : 0);
        p.any_passable = p.any_passable || pass;
    }
    for (size_t i = 0; i < g.instances.size(); ++i) {
        Axes a;
        const Instance& inst = g.instances[i];
        if (inst.material_id < s.materials.size()) {
            const Material& m = s.materials[inst.material_id];
            if (!(m.anisotropy != m.anisotropy || m.anisotropy <= 0.0f || m.is_emissive()) && inst.mesh < g.meshes.size()) {
                a.on = true;
                a.centre = inst.transform.point(g.meshes[inst.mesh].bounds.centroid());
                a.axis = normalize(inst.transform.vector(Vec3(0, 0, 1)));
                a.x_axis = normalize(inst.transform.vector(Vec3(1, 0, 0)));
            }
        }
        p.tangent_axes.push_back(a);
    }
    p.lights = Lights::make(s);
    return p;
}

// Ray counts and traversal statistics. `merged` (optional) is the scene's geometry with every
// identity instance's triangles in one reference-layout BVH8: each query is traced there too,
// only to count what a single tree of the reference's layout visits.
struct PathStats {
    uint64_t rays = 0, nearest = 0, any = 0;
    TraceStats trace, shadow, merged_trace, merged_shadow;
    const Geometry* merged = nullptr;
};

bool Prepared::shadow(const Scene& s, const Ray& ray, Rgb& pass, PathStats& st) const {
    const Geometry& geo = s.geometry;
    if (!any_passable) {
        bool blocked = (floor_mode == 1 && floor_t(ray, false) < F_INF) || (st.any += 1, geo.occluded(ray, false, &st.shadow));
        if (st.merged) st.merged->occluded(ray, false, &st.merged_shadow);
        pass = WHITE;
        return !blocked;
    }
    // walk: through the cut-outs and thin walls up to the first surface that stops the ray
    float floor = floor_mode == 1 ? floor_t(ray, false) : F_INF;
    Rgb keep = WHITE;
    Ray r = ray;
    float travelled = 0.0f, blocker = F_INF;
    bool done = false;
    for (uint32_t k = 0; k < 32 && !done; ++k) {  // MAX_SHADOW_CROSSINGS
        RayHit hit;
        st.nearest += 1;
        if (!geo.trace(r, false, hit, &st.trace)) { blocker = floor; done = true; break; }
        float t = travelled + hit.t;
        if (t >= floor) { blocker = floor; done = true; break; }
        if (!(hit.instance < passable.size() && passable[hit.instance])) { blocker = t; done = true; break; }
        Hit d;
        if (!geo.hit_details(r, hit, d)) { blocker = t; done = true; break; }
        Vec3 origin;
        keep = keep * straight_through(s, r, hit.instance, d, origin);
        if (rmax(rmax(keep.r, keep.g), keep.b) <= 0.0f) { keep = BLACK; blocker = t; done = true; break; }
        travelled += dot(origin - r.origin, r.dir);
        Ray next(origin, r.dir);
        next.t_max = ray.t_max - travelled;
        if (next.t_max != next.t_max || next.t_max <= next.t_min) { blocker = F_INF; done = true; break; }
        r = next;
    }
    if (!done) { keep = BLACK; blocker = travelled; }
    pass = keep;
    return blocker == F_INF && peak(keep) > 0.0f;
}

// One parameter perturbed for the adjoint's reference gradient, detached: sampling, light
// selection, MIS weights and roulette are those of the unperturbed scene, while what a path
// carries is evaluated with the perturbed value (the estimator the adjoint differentiates).
struct Perturb {
    int kind = 0;             // 1: a material's base colour (all channels at once), 2: its GGX alpha, 3: a light's power
    uint32_t index = 0;       // the material (kinds 1, 2) or the scene light (kind 3)
    Bsdf outside, inside;     // kinds 1, 2: the perturbed material's BSDFs
    Rgb sigma;                // kind 1: its medium's absorption per mm (when it has one)
    float light_ratio = 1.0f; // kind 3: perturbed power / power
};

// radiance_weighted (integrator/mod.rs:1140) for the scene features this subset reads. With
// `pert`, *out_pert receives the same path's radiance under the detached perturbation.
static void radiance(const Scene& scene, const Prepared& prep, const PixelSampler& sampler, Ray camera_ray, float su, float sv,
                     Rgb& out, float& alpha_out, PathStats& st, const Perturb* pert = nullptr, Rgb* out_pert = nullptr) {
    const Lights& lights = prep.lights;
    Ray ray = camera_ray;
    Rgb throughput = WHITE, sum = BLACK;
    Rgb thr_p = WHITE, sum_p = BLACK;  // under the perturbation
    const int only = pert && pert->kind == 3 ? (int)pert->index : -1;
    const float ratio = pert && pert->kind == 3 ? pert->light_ratio : 1.0f;
    uint32_t medium_material = 0;
    float alpha = 1.0f;
    bool has_pdf = false;
    float bsdf_pdf = 0.0f;
    Selection sampled_at = lights.select_by_flux(camera_ray.origin);
    uint32_t bounce = 0;
    bool primary = true;
    float offset = 0.0f;
    bool in_medium = false;
    uint32_t cutouts = 0;
    Rgb sigma;
    const Geometry& geo = scene.geometry;
    for (;;) {
        st.rays += 1;
        RayHit hit;
        st.nearest += 1;
        bool got = geo.trace(ray, primary, hit, &st.trace);
        if (st.merged) {
            RayHit unused;
            st.merged->trace(ray, primary, unused, &st.merged_trace);
        }
        float t_geometry = got ? hit.t : F_INF;
        float t_floor = prep.floor_t(ray, primary);
        float t_nearest = rmin(t_geometry, t_floor);
        if (in_medium && finite(t_nearest)) {
            Rgb bl(fexp(-sigma.r * t_nearest), fexp(-sigma.g * t_nearest), fexp(-sigma.b * t_nearest));
            throughput = throughput * bl;
            if (pert) {
                const bool mine = pert->kind == 1 && medium_material == pert->index;
                const Rgb& sg = mine ? pert->sigma : sigma;
                thr_p = thr_p * (mine ? Rgb(fexp(-sg.r * t_nearest), fexp(-sg.g * t_nearest), fexp(-sg.b * t_nearest)) : bl);
            }
        }
        const float* sp = has_pdf ? &bsdf_pdf : nullptr;
        Rgb part;
        Rgb crossed = lights.crossed_from(ray, t_nearest, sp, &sampled_at, offset, only, pert ? &part : nullptr);
        prep.add(sum, throughput * crossed, bounce >= 2);
        if (pert) prep.add(sum_p, thr_p * (crossed + part * (ratio - 1.0f)), bounce >= 2);
        if (t_nearest == F_INF) {
            if (primary && prep.background == 0) {
                Rgb seen = lights.escaped(ray.dir, nullptr, nullptr, only, pert ? &part : nullptr);
                float k = scene.camera.exterior;
                sum = sum + throughput * (k == 1.0f ? seen : seen * k);
                if (pert) {
                    Rgb seen_p = seen + part * (ratio - 1.0f);
                    sum_p = sum_p + thr_p * (k == 1.0f ? seen_p : seen_p * k);
                }
            } else if (primary && (prep.background == 1 || prep.background == 3)) {
                sum = sum + throughput * prep.backdrop(su, sv);
                if (pert) sum_p = sum_p + thr_p * prep.backdrop(su, sv);
            } else if (primary && prep.background == 2) {
                alpha = peak(crossed) > 0.0f ? 1.0f : 0.0f;
            } else {
                Rgb sky = lights.escaped(ray.dir, sp, &sampled_at, only, pert ? &part : nullptr);
                prep.add(sum, throughput * sky, bounce >= 2);
                if (pert) prep.add(sum_p, thr_p * (sky + part * (ratio - 1.0f)), bounce >= 2);
            }
            break;
        }
        // The surface: the floor, or an instance with its shading point (bevel.rs:232).
        Vec3 s_point, s_hit_point, s_normal, s_geometric;
        bool s_inst = false, s_outside = true, s_front = true;
        uint32_t inst = 0;
        if (t_floor < t_geometry) {
            Vec3 pp = ray.at(t_floor);
            Vec3 point(pp.x, pp.y, prep.floor_z);
            Vec3 n(0, 0, ray.dir.z < 0.0f ? 1.0f : -1.0f);
            s_point = point; s_hit_point = point; s_normal = n; s_geometric = n;
        } else {
            Hit d;
            if (!geo.hit_details(ray, hit, d)) break;
            Vec3 ng = d.geometric_normal;
            Vec3 normal = d.normal;
            if (dot(normal, ng) < 0.0f) normal = -normal;
            if (dot(normal, ray.dir) >= -1.0e-4f) normal = ng;
            s_point = geo.terminator_point(d);
            s_hit_point = d.point;
            s_normal = normal;
            s_geometric = ng;
            s_inst = true;
            inst = d.instance;
            s_outside = d.outside;
            s_front = d.front_face;
        }
        const Material* material = s_inst ? &prep.material(scene, inst) : nullptr;
        if (material && material->is_emissive()) {
            bool one_sided = (geo.instances[inst].flags & INSTANCE_ONE_SIDED) != 0;
            if (s_front || !one_sided) {
                // A BSDF-sampled ray that finds a mesh light weighs its emission against the light's
                // next-event sample; other emitters (and camera rays) weigh 1 (integrator/mod.rs:1556,
                // light.rs:1543).
                float weight = has_pdf ? lights.emitter_weight(inst, bsdf_pdf, sampled_at, offset + t_geometry, dot(s_geometric, ray.dir)) : 1.0f;
                prep.add(sum, throughput * material->radiance() * weight, bounce >= 2);
                if (pert) prep.add(sum_p, thr_p * material->radiance() * weight, bounce >= 2);
            }
            break;
        }
        // A cut-out lets the ray through with probability 1 - opacity (integrator/mod.rs:1571).
        if (material && material->opacity < 1.0f && cutouts < 64) {  // MAX_CUTOUTS
            float u = sampler.get1(cutout_dim(bounce, cutouts));
            cutouts += 1;
            if (u >= rmax(material->opacity, 0.0f)) {
                Vec3 o = offset_origin(s_hit_point, -s_geometric);
                offset += dot(o - ray.origin, ray.dir);
                ray = Ray(o, ray.dir);
                continue;
            }
        }
        if (bounce >= prep.max_depth) break;
        Bsdf bsdf = material ? Bsdf::surface(*material, s_outside) : prep.floor_bsdf;
        // the vertex's BSDF under the perturbation, when it is the perturbed material's
        const bool perturbed = pert && (pert->kind == 1 || pert->kind == 2) && material && s_inst &&
                               geo.instances[inst].material_id == pert->index;
        const Bsdf* bsdf_p = perturbed ? (s_outside ? &pert->outside : &pert->inside) : nullptr;
        Frame frame = prep.frame(s_inst, inst, s_point, s_normal);
        Vec3 wo = frame.to_local(-ray.dir);
        Vec3 ng = s_geometric;
        Vec3 origin = offset_origin(s_point, ng);
        uint32_t dims = bounce_dim(bounce);

        // Next-event estimation (integrator/mod.rs:1702).
        Selection selection = lights.select(s_point);
        float ul0, ul1;
        sampler.get2(dims + OFFSET_LIGHT, ul0, ul1);
        LightSample ls;
        float usel = sampler.get1(dims + OFFSET_LIGHT_SELECT);
        if (lights.sample_selected(selection, usel, ul0, ul1, ls)) {
            Vec3 wi = frame.to_local(ls.wi);
            Lobes lobes = ls.glossy ? Lobes::All : Lobes::Diffuse;
            Rgb f = bsdf.eval(wo, wi, lobes);
            if (peak(f) > 0.0f) {
                Vec3 from = wi.z < 0.0f ? offset_origin(s_hit_point, -ng) : origin;
                float distance = ls.distance;
                bool arrives = true;
                Rgb pass = WHITE;
                if (ls.shadow) {
                    st.rays += 1;
                    Ray sr(from, ls.wi);
                    if (finite(distance)) sr.t_max = distance * (1.0f - 1.0e-4f);
                    arrives = prep.shadow(scene, sr, pass, st);
                }
                if (arrives) {
                    float weight = (ls.delta || !ls.glossy) ? 1.0f : power_heuristic(ls.pdf, bsdf.pdf(wo, wi));
                    Rgb c = throughput * f * ls.radiance * (std::fabs(wi.z) * weight / ls.pdf);
                    if (!(pass == WHITE)) c = c * pass;
                    prep.add(sum, c, bounce >= 1);
                    if (pert) {
                        Rgb fp = bsdf_p ? bsdf_p->eval(wo, wi, lobes) : f;
                        Rgb lp = ls.source == only && only >= 0 ? ls.radiance * ratio : ls.radiance;
                        Rgb cp = thr_p * fp * lp * (std::fabs(wi.z) * weight / ls.pdf);
                        if (!(pass == WHITE)) cp = cp * pass;
                        prep.add(sum_p, cp, bounce >= 1);
                    }
                }
            }
        }
        // The next direction.
        float ub0, ub1;
        sampler.get2(dims + OFFSET_BSDF, ub0, ub1);
        BsdfSample bs;
        if (!bsdf.sample(wo, ub0, ub1, bs)) break;
        bool transmitted = bs.wi.z < 0.0f;
        Vec3 wi = bs.straight ? ray.dir : normalize(frame.to_world(bs.wi));
        if (transmitted) {
            if (dot(wi, ng) >= 0.0f) break;
        } else if (dot(wi, ng) <= 0.0f) {
            break;
        }
        throughput = throughput * bs.weight;
        if (pert) {
            Rgb k = bs.weight;
            if (bsdf_p && !bs.straight) {  // the sample's weight f / pdf with f perturbed, pdf held
                Rgb f = bsdf.eval(wo, bs.wi, Lobes::All), fp = bsdf_p->eval(wo, bs.wi, Lobes::All);
                k = Rgb(f.r > 0.0f ? k.r * (fp.r / f.r) : k.r, f.g > 0.0f ? k.g * (fp.g / f.g) : k.g, f.b > 0.0f ? k.b * (fp.b / f.b) : k.b);
            }
            thr_p = thr_p * k;
        }
        if (bounce >= 2) {
            float survive = rclamp(peak(throughput), 0.05f, 1.0f);
            if (sampler.get1(dims + OFFSET_ROULETTE) >= survive) break;
            throughput = throughput / survive;
            if (pert) thr_p = thr_p / survive;
        }
        float pk = peak(throughput);
        if (!(pk > 0.0f && finite(pk))) break;
        Vec3 next_origin = transmitted ? offset_origin(s_hit_point, -ng) : origin;
        if (bs.straight) {
            offset += dot(next_origin - ray.origin, ray.dir);
        } else {
            has_pdf = true;
            bsdf_pdf = bs.pdf;
            sampled_at = selection;
            primary = false;
            offset = 0.0f;
            if (transmitted) {
                if (s_outside && material && s_inst) {
                    uint32_t mid = geo.instances[inst].material_id;
                    in_medium = mid < prep.has_medium.size() && prep.has_medium[mid];
                    if (in_medium) sigma = prep.media[mid];
                    medium_material = mid;
                } else {
                    in_medium = false;
                }
            }
        }
        ray = Ray(next_origin, wi);
        bounce += 1;
    }
    out = sum;
    alpha_out = alpha;
    if (out_pert) *out_pert = sum_p;
}

// The inverse CDF of the Blackman-Harris window (F. J. Harris, Proc. IEEE 66, 1978: a0 - a1 cos 2pi t
// + a2 cos 4pi t - a3 cos 6pi t) three pixels wide, at the 256 points u = q(i / 255), q(s) = 2 s^2
// below one half and 1 - 2 (1 - s)^2 above: each by 100 bisections of the window's integral in
// f64, rounded to f32 (pixel_filter.rs:56-95 and the generator of its table test).
static const float* blackman_harris_table() {
    static float table[256];
    static bool ready = false;
    if (!ready) {
        const double a0 = 0.35875, a1 = 0.48829, a2 = 0.14128, a3 = 0.01168, pi = 3.14159265358979323846, r = 1.5;
        auto cdf = [&](double x) {
            double t = (x + r) / (2.0 * r);
            t = t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t);
            return (a0 * t - a1 * std::sin(2.0 * pi * t) / (2.0 * pi) + a2 * std::sin(4.0 * pi * t) / (4.0 * pi) -
                    a3 * std::sin(6.0 * pi * t) / (6.0 * pi)) /
                   a0;
        };
        for (int i = 0; i < 256; ++i) {
            double sq = (double)i / 255.0;
            double u = sq < 0.5 ? 2.0 * sq * sq : 1.0 - 2.0 * (1.0 - sq) * (1.0 - sq);
            double a = -r, b = r;
            for (int k = 0; k < 100; ++k) {
                double m = 0.5 * (a + b);
                if (cdf(m) < u) a = m;
                else b = m;
            }
            table[i] = (float)(0.5 * (a + b));
        }
        ready = true;
    }
    return table;
}
static float filter_offset(uint32_t filter, float u) {  // pixel_filter.rs:103
    if (filter == 1) return 0.5f;
    if (filter == 2) return 0.5f + (u < 0.5f ? std::sqrt(2.0f * u) - 1.0f : 1.0f - std::sqrt(2.0f - 2.0f * u));
    if (filter == 3) {  // pixel_filter.rs:125: the table interpolated at s = q^-1(u)
        const float* t = blackman_harris_table();
        float s = u < 0.5f ? std::sqrt(0.5f * u) : 1.0f - std::sqrt(0.5f - 0.5f * u);
        float f = rclamp(s * 255.0f, 0.0f, 255.0f);
        size_t i = (size_t)f < 254 ? (size_t)f : 254;
        float w = f - (float)i;
        return 0.5f + (t[i] + (t[i + 1] - t[i]) * w);
    }
    return u;
}

// The camera ray of sample `index` of pixel (x, y) (render.rs:79 camera_sample_weighted); (u, v)
// its screen position.
static Ray sample_ray(const Scene& scene, const PixelSampler& sampler, uint32_t x, uint32_t y, float& u, float& v) {
    uint32_t width = scene.render.width ? scene.render.width : 1, height = scene.render.height ? scene.render.height : 1;
    float aspect = (float)width / (float)height;
    float du, dv;
    sampler.get2(DIM_CAMERA, du, dv);
    du = filter_offset(scene.render.pixel_filter, du);
    dv = filter_offset(scene.render.pixel_filter, dv);
    u = ((float)x + du) / (float)width;
    v = ((float)y + dv) / (float)height;
    float lx = 0.0f, ly = 0.0f;
    if (scene.camera.lens_radius() > 0.0f) {
        float a, b;
        sampler.get2(DIM_LENS, a, b);
        concentric_disk(a, b, lx, ly);
    }
    return scene.camera.generate_ray(aspect, u, v, lx, ly);
}

// camera_sample_weighted (render.rs:79) and the shade of render_tile_traced (render.rs:388).
// Sample indices from `split_b` on are scrambled with the seed's complement (the decorrelated
// adjoint's second half); renders leave it at 0xffffffff.
static void shade_pixel(const Scene& scene, const Prepared& prep, uint32_t x, uint32_t y, uint32_t index, Rgb& c,
                        float& alpha, PathStats& st, const Perturb* pert = nullptr, Rgb* c_pert = nullptr,
                        uint32_t split_b = 0xffffffffu) {
    uint32_t width = scene.render.width ? scene.render.width : 1, height = scene.render.height ? scene.render.height : 1;
    float aspect = (float)width / (float)height;
    PixelSampler sampler(index >= split_b ? ~scene.render.seed : scene.render.seed, x, y, index);
    float du, dv;
    sampler.get2(DIM_CAMERA, du, dv);
    du = filter_offset(scene.render.pixel_filter, du);
    dv = filter_offset(scene.render.pixel_filter, dv);
    float u = ((float)x + du) / (float)width;
    float v = ((float)y + dv) / (float)height;
    float lx = 0.0f, ly = 0.0f;
    if (scene.camera.lens_radius() > 0.0f) {
        float a, b;
        sampler.get2(DIM_LENS, a, b);
        concentric_disk(a, b, lx, ly);
    }
    Ray ray = scene.camera.generate_ray(aspect, u, v, lx, ly);
    radiance(scene, prep, sampler, ray, rclamp(u, 0.0f, 1.0f), rclamp(v, 0.0f, 1.0f), c, alpha, st, pert, c_pert);
    // A panoramic camera's sample where it sees nothing brings no light (scene/mod.rs:338: its
    // weight is black; render.rs:465 multiplies the radiance by it).
    if (scene.camera.panoramic() && !(ray.t_max > 0.0f)) {
        c = c * BLACK;
        if (c_pert) *c_pert = *c_pert * BLACK;
    }
}

// The exact passes of a centre ray (passes.rs:168) that the edge mask compares: part and
// material ids (instance or material + 1, FLOOR_ID for the floor, 0 for the background) and the
// depth along the view axis.
struct Exact { uint32_t part = 0, material = 0; float depth = F_INF; Vec3 normal; };
constexpr uint32_t FLOOR_ID = 0xffffffffu;
// first_hit (integrator/mod.rs:911) for the albedo pass (passes.rs:209 albedo_of): the base colour
// of the material of what the ray met (the default material's for an index out of range), the
// floor's colour, black for the background. `covers` (may be null) gets passes.rs:221
// coverage_of: 1 for FirstHit::Surface, 0 for the floor and the background (a light panel too).
static Rgb first_albedo(const Scene& scene, const Prepared& prep, const Ray& ray, float* covers = nullptr) {
    if (covers) *covers = 0.0f;
    RayHit hit;
    bool got = scene.geometry.trace(ray, true, hit, nullptr);
    float t_geometry = got ? hit.t : F_INF;
    float t_floor = prep.floor_t(ray, true);
    float t_nearest = rmin(t_geometry, t_floor);
    if (t_nearest == F_INF || prep.lights.camera_sees_panel(ray, t_nearest)) return BLACK;
    if (t_floor < t_geometry) return scene.floor.color;
    Hit d;
    if (!scene.geometry.hit_details(ray, hit, d)) return BLACK;
    if (covers) *covers = 1.0f;
    return prep.material(scene, d.instance).base_color;
}
// render.rs:503 centre_ray and integrator/mod.rs:911 first_hit, as Exact::of reads them.
static Exact centre_exact(const Scene& scene, const Prepared& prep, uint32_t x, uint32_t y) {
    uint32_t width = scene.render.width ? scene.render.width : 1, height = scene.render.height ? scene.render.height : 1;
    float aspect = (float)width / (float)height;
    Ray ray = scene.camera.generate_ray(aspect, ((float)x + 0.5f) / (float)width, ((float)y + 0.5f) / (float)height, 0.0f, 0.0f);
    RayHit hit;
    bool got = scene.geometry.trace(ray, true, hit, nullptr);
    float t_geometry = got ? hit.t : F_INF;
    float t_floor = prep.floor_t(ray, true);
    float t_nearest = rmin(t_geometry, t_floor);
    Exact e;
    if (t_nearest == F_INF || prep.lights.camera_sees_panel(ray, t_nearest)) return e;
    float t;
    if (t_floor < t_geometry) {
        e.part = e.material = FLOOR_ID;
        e.normal = Vec3(0.0f, 0.0f, ray.dir.z < 0.0f ? 1.0f : -1.0f);
        t = t_floor;
    } else {
        Hit d;
        if (!scene.geometry.hit_details(ray, hit, d)) return e;
        e.normal = d.normal;
        e.part = d.instance + 1;
        uint32_t m = scene.geometry.instances[d.instance].material_id;
        e.material = m < scene.materials.size() ? m + 1 : 0;
        t = d.t;
    }
    Vec3 forward, right, upv;
    scene.camera.basis(forward, right, upv);
    // passes.rs:191: along the view axis; a panorama has no axis for what it sees: the distance.
    e.depth = scene.camera.panoramic() ? t * length(ray.dir) : t * dot(ray.dir, forward) + dot(ray.origin - scene.camera.position, forward);
    return e;
}
// EdgeMask::of (pixel_filter.rs:175) for the whole image (the same for any tile cut): a pixel is
// an edge when one of its neighbours inside the image sees another part, another material or a
// depth more than 2 % away through its centre.
static std::vector<uint8_t> edge_mask(const Scene& scene, const Prepared& prep) {
    uint32_t w = scene.render.width, h = scene.render.height;
    std::vector<Exact> c((size_t)w * h);
    for (uint32_t y = 0; y < h; ++y)
        for (uint32_t x = 0; x < w; ++x) c[(size_t)y * w + x] = centre_exact(scene, prep, x, y);
    auto differs = [](const Exact& a, const Exact& b) {
        return a.part != b.part || a.material != b.material || std::fabs(a.depth - b.depth) > 0.02f * rmin(a.depth, b.depth);
    };
    std::vector<uint8_t> edge((size_t)w * h, 0);
    for (uint32_t y = 0; y < h; ++y)
        for (uint32_t x = 0; x < w; ++x) {
            bool is = false;
            for (uint32_t ny = y ? y - 1 : 0; ny < std::min(y + 2, h); ++ny)
                for (uint32_t nx = x ? x - 1 : 0; nx < std::min(x + 2, w); ++nx) is |= differs(c[(size_t)y * w + x], c[(size_t)ny * w + nx]);
            edge[(size_t)y * w + x] = is ? 1 : 0;
        }
    return edge;
}

struct Film {
    uint32_t ox, oy, w, h;
    std::vector<float> rgb, weight, alpha, lum2;
    Film(uint32_t x, uint32_t y, uint32_t ww, uint32_t hh)
        : ox(x), oy(y), w(ww), h(hh), rgb((size_t)ww * hh * 3), weight((size_t)ww * hh), alpha((size_t)ww * hh), lum2((size_t)ww * hh) {}
    void splat(uint32_t x, uint32_t y, Rgb c, float a) {  // image.rs:82
        if (x < ox || y < oy || x - ox >= w || y - oy >= h) return;
        size_t i = (size_t)(y - oy) * w + (x - ox);
        rgb[3 * i] += c.r;
        rgb[3 * i + 1] += c.g;
        rgb[3 * i + 2] += c.b;
        weight[i] += 1.0f;
        alpha[i] += a;
        float l = c.luminance();
        lum2[i] += l * l;
    }
};

// render_tile_traced (render.rs:388) into `film`, one sample index. `edges` (one byte per image
// pixel, or empty): an edge pixel renders k = edge_supersample samples, indices index k .. index k +
// k - 1, and splats their mean (render.rs:477).
static void render_tile(const Scene& scene, const Prepared& prep, const std::vector<uint8_t>& edges, uint32_t tx, uint32_t ty,
                        uint32_t tw, uint32_t th, uint32_t index, Film& film, PathStats& st) {
    uint32_t x_end = std::min<uint64_t>((uint64_t)tx + tw, scene.render.width);
    uint32_t y_end = std::min<uint64_t>((uint64_t)ty + th, scene.render.height);
    const uint32_t k = scene.render.edge_supersample < 1 ? 1 : (scene.render.edge_supersample > 16 ? 16 : scene.render.edge_supersample);
    for (uint32_t y = ty; y < y_end; ++y)
        for (uint32_t x = tx; x < x_end; ++x) {
            Rgb c;
            float a;
            if (k <= 1 || edges.empty() || !edges[(size_t)y * scene.render.width + x]) {
                shade_pixel(scene, prep, x, y, index, c, a, st);
                film.splat(x, y, c * WHITE, a);
                continue;
            }
            Rgb sum = BLACK;
            float coverage = 0.0f;
            for (uint32_t j = 0; j < k; ++j) {
                shade_pixel(scene, prep, x, y, index * k + j, c, a, st);
                sum = sum + c * WHITE;
                coverage += a;
            }
            float inv = 1.0f / (float)k;
            film.splat(x, y, sum * inv, coverage * inv);
        }
}

struct Loaded {
    Scene scene;
    Prepared prep;
    std::vector<uint8_t> edges;  // the edge mask when edge_supersample > 1, else empty
    std::unique_ptr<Geometry> merged;  // statistics only (see PathStats)
};

// The scene's geometry with the triangles of all identity instances in one mesh (world space,
// one reference-layout BVH8); transformed instances keep their own meshes and transforms.
static void build_merged(const Geometry& g, Geometry& out) {
    std::vector<Vec3> pos;
    std::vector<uint32_t> idx;
    std::vector<Mesh> meshes(1);
    std::vector<Instance> insts(1);
    for (size_t i = 0; i < g.instances.size(); ++i) {
        const Instance& in = g.instances[i];
        if (!g.prepared[i].active) continue;
        const Mesh& m = g.meshes[in.mesh];
        if (g.prepared[i].identity) {
            uint32_t base = (uint32_t)pos.size();
            pos.insert(pos.end(), m.positions.begin(), m.positions.end());
            for (uint32_t k : m.indices) idx.push_back(base + k);
        } else {
            Instance copy = in;
            copy.mesh = (uint32_t)meshes.size();
            meshes.push_back(m);
            insts.push_back(copy);
        }
    }
    Mesh::make(meshes[0], pos, {}, idx, 0);
    Geometry::make(out, std::move(meshes), std::move(insts));
}

}  // namespace orc

using namespace orc;

namespace {
std::mutex g_mu;
std::vector<std::unique_ptr<Loaded>> g_scenes;
std::string g_error;
Loaded* get(uint32_t h) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (h == 0 || h > g_scenes.size()) return nullptr;
    return g_scenes[h - 1].get();
}
}  // namespace

// Runs fn(begin, end, worker) over [0, n) in `threads` contiguous chunks (0: the host's cores).
template <class F>
static void parallel_chunks(uint32_t n, uint32_t threads, F fn) {
    if (threads == 0) threads = std::max(1u, std::thread::hardware_concurrency());
    threads = std::max(1u, std::min(threads, n / 16 + 1));
    std::vector<std::thread> pool;
    const uint32_t per = (n + threads - 1) / threads;
    for (uint32_t t = 0; t < threads; ++t) {
        const uint32_t b = std::min(n, t * per), e = std::min(n, b + per);
        pool.emplace_back([=]() { fn(b, e, t); });
    }
    for (auto& th : pool) th.join();
}

extern "C" {

// Loads an RSB scene; 0 on error (orc_error gives the message).
uint32_t orc_scene_load(const uint8_t* bytes, uint32_t len) {
    if (!bytes) return 0;
    auto l = std::make_unique<Loaded>();
    std::string err;
    if (!read_rsb(bytes, len, l->scene, err)) {
        std::lock_guard<std::mutex> lk(g_mu);
        g_error = err;
        return 0;
    }
    l->prep = Prepared::make(l->scene);
    if (l->scene.render.edge_supersample > 1) l->edges = edge_mask(l->scene, l->prep);
    std::lock_guard<std::mutex> lk(g_mu);
    g_error.clear();
    for (size_t i = 0; i < g_scenes.size(); ++i)
        if (!g_scenes[i]) { g_scenes[i] = std::move(l); return (uint32_t)i + 1; }
    g_scenes.push_back(std::move(l));
    return (uint32_t)g_scenes.size();
}
uint32_t orc_error(char* out, uint32_t cap) {
    std::lock_guard<std::mutex> lk(g_mu);
    uint32_t n = (uint32_t)g_error.size();
    if (out && cap) { uint32_t k = n < cap - 1 ? n : cap - 1; std::memcpy(out, g_error.data(), k); out[k] = 0; }
    return n;
}
uint32_t orc_scene_free(uint32_t h) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (h == 0 || h > g_scenes.size() || !g_scenes[h - 1]) return 1;
    g_scenes[h - 1].reset();
    return 0;
}
// Scene facts: width, height, seed, max_depth, instance count, triangle count (instanced).
// out8: width, height, seed, max depth, instances, triangles, materials, scene lights.
uint32_t orc_scene_info(uint32_t h, uint32_t* out6) {
    Loaded* l = get(h);
    if (!l || !out6) return 1;
    out6[6] = (uint32_t)l->scene.materials.size();
    out6[7] = (uint32_t)l->scene.lights.size();
    out6[0] = l->scene.render.width;
    out6[1] = l->scene.render.height;
    out6[2] = l->scene.render.seed;
    out6[3] = l->prep.max_depth;
    out6[4] = (uint32_t)l->scene.geometry.instances.size();
    uint64_t tris = 0;
    for (const Instance& in : l->scene.geometry.instances) tris += l->scene.geometry.meshes[in.mesh].triangle_count();
    out6[5] = (uint32_t)tris;
    return 0;
}

// Film accumulation over a region, samples [first, first + count) per pixel in order, tiles of
// `tile` pixels claimed by `threads` workers (rt-cli/src/lib.rs:266-368). Outputs are the film's
// sums: rgb (3 per pixel), weight, alpha, lum2. Returns the ray count; stats7 (may be null) gets
// rays; nearest-hit queries, their reference-BVH8 inner-node visits and packet tests; any-hit
// queries, their node visits and packet tests; then (after orc_enable_merged_stats) the node
// visits and packet tests of the same nearest and any-hit queries in the merged tree.
uint64_t orc_render_film(uint32_t h, uint32_t x0, uint32_t y0, uint32_t w, uint32_t hgt, uint32_t first, uint32_t count,
                         uint32_t tile, uint32_t threads, float* rgb, float* weight, float* alpha, float* lum2,
                         uint64_t* stats11) {
    Loaded* l = get(h);
    if (!l || !rgb || w == 0 || hgt == 0) return 0;
    if (tile == 0) tile = 32;
    if (threads == 0) threads = 1;
    std::vector<uint32_t> tiles;
    for (uint32_t y = 0; y < hgt; y += tile)
        for (uint32_t x = 0; x < w; x += tile) { tiles.push_back(x); tiles.push_back(y); }
    std::atomic<size_t> next(0);
    std::atomic<uint64_t> rays(0), nq(0), nodes(0), packets(0), aq(0), anodes(0), apackets(0);
    std::atomic<uint64_t> mnodes(0), mpackets(0), manodes(0), mapackets(0);
    auto worker = [&]() {
        PathStats st;
        st.merged = l->merged.get();
        for (;;) {
            size_t t = next.fetch_add(1);
            if (t >= tiles.size() / 2) break;
            uint32_t tx = tiles[2 * t], ty = tiles[2 * t + 1];
            uint32_t tw = std::min(tile, w - tx), th = std::min(tile, hgt - ty);
            Film film(x0 + tx, y0 + ty, tw, th);
            for (uint32_t s = 0; s < count; ++s) render_tile(l->scene, l->prep, l->edges, x0 + tx, y0 + ty, tw, th, first + s, film, st);
            for (uint32_t yy = 0; yy < th; ++yy)
                for (uint32_t xx = 0; xx < tw; ++xx) {
                    size_t i = (size_t)yy * tw + xx, o = (size_t)(ty + yy) * w + (tx + xx);
                    for (int c = 0; c < 3; ++c) rgb[3 * o + c] += film.rgb[3 * i + c];
                    if (weight) weight[o] += film.weight[i];
                    if (alpha) alpha[o] += film.alpha[i];
                    if (lum2) lum2[o] += film.lum2[i];
                }
        }
        rays += st.rays;
        nq += st.nearest;
        nodes += st.trace.nodes;
        packets += st.trace.packets;
        aq += st.any;
        anodes += st.shadow.nodes;
        apackets += st.shadow.packets;
        mnodes += st.merged_trace.nodes;
        mpackets += st.merged_trace.packets;
        manodes += st.merged_shadow.nodes;
        mapackets += st.merged_shadow.packets;
    };
    std::vector<std::thread> pool;
    for (uint32_t i = 0; i < threads; ++i) pool.emplace_back(worker);
    for (auto& t : pool) t.join();
    if (stats11) {
        uint64_t v[11] = {rays, nq, nodes, packets, aq, anodes, apackets, mnodes, mpackets, manodes, mapackets};
        std::memcpy(stats11, v, sizeof(v));
    }
    return rays;
}

// rt_render_tile_passes (rt-wasm/src/lib.rs:484, render.rs:515 render_tile_exact): the exact passes
// of the rectangle's centre rays, background outside the image: normal (3 a pixel), depth, part
// id and material id (each may be null).
uint32_t orc_render_passes(uint32_t h, uint32_t x0, uint32_t y0, uint32_t w, uint32_t hh, float* normal, float* depth, uint32_t* part,
                           uint32_t* material) {
    Loaded* l = get(h);
    if (!l) return 1;
    const uint32_t W = l->scene.render.width, H = l->scene.render.height;
    for (uint32_t y = 0; y < hh; ++y)
        for (uint32_t x = 0; x < w; ++x) {
            const size_t i = (size_t)y * w + x;
            Exact e;
            if ((uint64_t)x0 + x < W && (uint64_t)y0 + y < H) e = centre_exact(l->scene, l->prep, x0 + x, y0 + y);
            if (normal) { normal[3 * i] = e.normal.x; normal[3 * i + 1] = e.normal.y; normal[3 * i + 2] = e.normal.z; }
            if (depth) depth[i] = e.depth;
            if (part) part[i] = e.part;
            if (material) material[i] = e.material;
        }
    return 0;
}

// rt_render_tile_albedo (rt-wasm/src/lib.rs:510, render.rs:590): the albedo of sample `index` of
// the rectangle's pixels, 3 floats a pixel (0 outside the image); an edge pixel gives the mean of
// its k sub-samples.
// render.rs:590 render_tile_albedo_traced, its alpha plane (rt-wasm lib.rs:537
// render_tile_alpha_sample): the coverage of sample `index` of each pixel of the rectangle, an
// edge pixel's the mean over its k sub-samples (summed in order, times 1/k), 0 outside the image.
uint32_t orc_render_alpha(uint32_t h, uint32_t x0, uint32_t y0, uint32_t w, uint32_t hh, uint32_t index, float* out) {
    Loaded* l = get(h);
    if (!l || !out) return 1;
    const Scene& sc = l->scene;
    const uint32_t W = sc.render.width, H = sc.render.height;
    const uint32_t k = sc.render.edge_supersample < 1 ? 1 : (sc.render.edge_supersample > 16 ? 16 : sc.render.edge_supersample);
    for (uint32_t y = 0; y < hh; ++y)
        for (uint32_t x = 0; x < w; ++x) {
            const size_t i = (size_t)y * w + x;
            float a = 0.0f;
            const uint32_t px = x0 + x, py = y0 + y;
            if ((uint64_t)x0 + x < W && (uint64_t)y0 + y < H) {
                const bool edge = k > 1 && !l->edges.empty() && l->edges[(size_t)py * W + px];
                float u, v;
                if (!edge) {
                    first_albedo(sc, l->prep, sample_ray(sc, PixelSampler(sc.render.seed, px, py, index), px, py, u, v), &a);
                } else {
                    float covered = 0.0f;
                    for (uint32_t j = 0; j < k; ++j) {
                        float c = 0.0f;
                        first_albedo(sc, l->prep, sample_ray(sc, PixelSampler(sc.render.seed, px, py, index * k + j), px, py, u, v), &c);
                        covered += c;
                    }
                    a = covered * (1.0f / (float)k);
                }
            }
            out[i] = a;
        }
    return 0;
}

uint32_t orc_render_albedo(uint32_t h, uint32_t x0, uint32_t y0, uint32_t w, uint32_t hh, uint32_t index, float* out) {
    Loaded* l = get(h);
    if (!l || !out) return 1;
    const Scene& sc = l->scene;
    const uint32_t W = sc.render.width, H = sc.render.height;
    const uint32_t k = sc.render.edge_supersample < 1 ? 1 : (sc.render.edge_supersample > 16 ? 16 : sc.render.edge_supersample);
    for (uint32_t y = 0; y < hh; ++y)
        for (uint32_t x = 0; x < w; ++x) {
            const size_t i = (size_t)y * w + x;
            Rgb a = BLACK;
            const uint32_t px = x0 + x, py = y0 + y;
            if ((uint64_t)x0 + x < W && (uint64_t)y0 + y < H) {
                const bool edge = k > 1 && !l->edges.empty() && l->edges[(size_t)py * W + px];
                float u, v;
                if (!edge) {
                    a = first_albedo(sc, l->prep, sample_ray(sc, PixelSampler(sc.render.seed, px, py, index), px, py, u, v));
                } else {
                    Rgb sum = BLACK;
                    for (uint32_t j = 0; j < k; ++j)
                        sum = sum + first_albedo(sc, l->prep, sample_ray(sc, PixelSampler(sc.render.seed, px, py, index * k + j), px, py, u, v));
                    a = sum * (1.0f / (float)k);
                }
            }
            out[3 * i] = a.r; out[3 * i + 1] = a.g; out[3 * i + 2] = a.b;
        }
    return 0;
}

// E10 (adaptive/tests.rs:294 adaptive_film, a scene without photon maps): renders scene `h`
// adaptively, at most `cap` samples a pixel (0: none), in passes of `pass` samples cut at the
// rounds, straight into one whole-image film: each active block renders its samples of the pass
// in index order (render.rs:352 render_block). The blocks of a pass are shared by `threads`
// workers; a block's pixels are its own, so any split gives the same film. Outputs the film's
// sums, each block's samples (counts, row by row) and state4 = the fewest and the most samples of
// a pixel, the decisions taken and the rays traced (low 32 bits). 0, or 1 for a bad handle.
uint32_t orc_adaptive_film(uint32_t h, uint32_t cap, uint32_t pass, uint32_t threads, float* rgb, float* weight, float* alpha,
                           float* lum2, uint32_t* counts, uint32_t* state4) {
    Loaded* l = get(h);
    if (!l || !rgb || !weight || !alpha || !lum2 || !counts || !state4) return 1;
    const RenderSettings& rs = l->scene.render;
    if (pass == 0) pass = AD_ROUND;
    if (threads == 0) threads = 1;
    Film film(0, 0, rs.width, rs.height);
    Adaptive ad(rs.width, rs.height, rs.exposure_ev, rs.noise_threshold, cap);
    std::vector<BlockWork> work;
    uint32_t decisions = 0;
    std::atomic<uint64_t> rays(0);
    for (;;) {
        if (ad.left() == 0) {
            ad.decide(film.rgb.data(), 3, film.lum2.data());
            ++decisions;
            if (ad.converged()) break;
        }
        const uint32_t count = std::min(pass, ad.left());
        ad.work(0, 0, rs.width, rs.height, count, work);
        std::atomic<size_t> next(0);
        auto worker = [&]() {
            PathStats st;
            for (;;) {
                const size_t i = next.fetch_add(1);
                if (i >= work.size()) break;
                const BlockWork& wk = work[i];
                for (uint32_t j = 0; j < wk.count; ++j)
                    render_tile(l->scene, l->prep, l->edges, wk.x, wk.y, wk.w, wk.h, wk.first + j, film, st);
            }
            rays += st.rays;
        };
        std::vector<std::thread> pool;
        for (uint32_t i = 0; i < threads; ++i) pool.emplace_back(worker);
        for (auto& t : pool) t.join();
        ad.advance(count);
    }
    const size_t n = (size_t)rs.width * rs.height;
    std::memcpy(rgb, film.rgb.data(), n * 12);
    std::memcpy(weight, film.weight.data(), n * 4);
    std::memcpy(alpha, film.alpha.data(), n * 4);
    std::memcpy(lum2, film.lum2.data(), n * 4);
    std::memcpy(counts, ad.counts.data(), ad.counts.size() * 4);
    ad.min_max(state4[0], state4[1]);
    state4[2] = decisions;
    state4[3] = (uint32_t)rays.load();
    return 0;
}

// Also counts every query's visits in a single reference-layout BVH8 over the identity
// instances' triangles (stats11[7..10] of orc_render_film); builds that tree once.
uint32_t orc_enable_merged_stats(uint32_t h) {
    Loaded* l = get(h);
    if (!l) return 1;
    if (!l->merged) {
        l->merged = std::make_unique<Geometry>();
        build_merged(l->scene.geometry, *l->merged);
    }
    return 0;
}

// One sample of each pixel of a tile as `rt_render_tile` gives it: w*h*3 radiance (resolved
// one-sample film), zero outside the image. Returns the ray count.
uint64_t orc_render_tile(uint32_t h, uint32_t x, uint32_t y, uint32_t w, uint32_t hgt, uint32_t sample, float* out_rgb,
                         float* out_alpha) {
    Loaded* l = get(h);
    if (!l || !out_rgb) return 0;
    Film film(x, y, w, hgt);
    PathStats st;
    render_tile(l->scene, l->prep, l->edges, x, y, w, hgt, sample, film, st);
    for (size_t i = 0; i < (size_t)w * hgt; ++i) {
        float wt = film.weight[i];
        float inv = wt > 0.0f ? 1.0f / wt : 0.0f;
        for (int c = 0; c < 3; ++c) out_rgb[3 * i + c] = wt > 0.0f ? film.rgb[3 * i + c] * inv : 0.0f;
        if (out_alpha) out_alpha[i] = wt > 0.0f ? film.alpha[i] * inv : 0.0f;
    }
    return st.rays;
}

// The adjoint's reference gradient on the CPU: the loss of the film of samples [first, first +
// count) of the rectangle (x0, y0, w, hgt) against `target` (w hgt 3 floats: mean over pixels and
// channels of (film - target)^2, summed in double), and its gradient with respect to every
// material's base colour (R, G, B) and GGX alpha and every scene light's power (grads: 4 per
// material, then one per light), for the estimator the device adjoint differentiates: detached
// sampling, and with two halves of the samples (count >= 2) each half's derivative weighted by
// the other half's residual (the derivative of the mean over pixels and channels of
// (mean_A - target)(mean_B - target)), half B drawn with the seed's complement as the device
// draws it; with one sample or `correlated`, of the loss itself. Each parameter's
// derivative is a central difference of the detached estimator (base colour and alpha +- 1e-3,
// as the device's BSDF differences; a light's power +- 1e-3 of itself), every sum in double.
// Returns 0, or 1 for a bad handle or argument.
uint32_t orc_adjoint_reference(uint32_t h, uint32_t x0, uint32_t y0, uint32_t w, uint32_t hgt, uint32_t first, uint32_t count,
                               uint32_t correlated, const float* target, uint32_t threads, double* grads, double* loss) {
    Loaded* l = get(h);
    if (!l || !target || !grads || !loss || w == 0 || hgt == 0 || count == 0) return 1;
    const Scene& sc = l->scene;
    const size_t npix = (size_t)w * hgt;
    const uint32_t nm = (uint32_t)sc.materials.size(), nl = (uint32_t)sc.lights.size();
    const uint32_t half = correlated ? 0 : count / 2;  // 0: one estimate from all samples
    // Per pixel and channel: the sums of halves A (samples before first + half) and B.
    auto render = [&](const Perturb* pert, std::vector<double>& sa, std::vector<double>& sb, std::vector<float>* film) {
        sa.assign(3 * npix, 0.0);
        sb.assign(3 * npix, 0.0);
        if (film) film->assign(3 * npix, 0.0f);
        parallel_chunks((uint32_t)npix, threads, [&](uint32_t b, uint32_t e, uint32_t) {
            for (uint32_t p = b; p < e; ++p) {
                const uint32_t px = x0 + p % w, py = y0 + p / w;
                float fr = 0.0f, fg = 0.0f, fb = 0.0f;
                for (uint32_t k = 0; k < count; ++k) {
                    PathStats st;
                    Rgb c, cp;
                    float a;
                    shade_pixel(sc, l->prep, px, py, first + k, c, a, st, pert, &cp, half > 0 ? first + half : 0xffffffffu);
                    const Rgb& v = pert ? cp : c;
                    double* acc = (half > 0 && k >= half) ? &sb[3 * p] : &sa[3 * p];
                    acc[0] += v.r; acc[1] += v.g; acc[2] += v.b;
                    fr = fr + c.r; fg = fg + c.g; fb = fb + c.b;
                }
                if (film) { (*film)[3 * p] = fr; (*film)[3 * p + 1] = fg; (*film)[3 * p + 2] = fb; }
            }
        });
    };
    std::vector<double> sa, sb, pa, pb, ma, mb;
    std::vector<float> film;
    render(nullptr, sa, sb, &film);
    // the loss, and each half's weights: d loss / d (its mean) per pixel and channel
    const double norm = 3.0 * (double)npix;
    std::vector<double> wa(3 * npix), wb(3 * npix);
    double lsum = 0.0;
    const float inv = 1.0f / (float)count;
    for (size_t i = 0; i < 3 * npix; ++i) {
        const double t = target[i];
        const double e = (double)(film[i] * inv) - t;
        lsum += e * e;
        if (half == 0) {
            wa[i] = 2.0 * e / norm;
            wb[i] = 0.0;
        } else {
            wa[i] = (sb[i] / (double)(count - half) - t) / norm;  // A's derivative takes B's residual
            wb[i] = (sa[i] / (double)half - t) / norm;
        }
    }
    *loss = lsum / norm;
    const double na = half == 0 ? (double)count : (double)half, nb = (double)(count - half);
    // sum over pixels of w . (mean_plus - mean_minus) per channel
    auto delta = [&](int c) {
        double g = 0.0;
        for (size_t p = 0; p < npix; ++p) {
            const size_t i = 3 * p + c;
            g += wa[i] * (pa[i] - ma[i]) / na;
            if (half > 0) g += wb[i] * (pb[i] - mb[i]) / nb;
        }
        return g;
    };
    const float hm = 1.0e-3f;
    for (uint32_t m = 0; m < nm; ++m) {
        for (int kind = 1; kind <= 2; ++kind) {
            Perturb plus, minus;
            for (int sgn = 0; sgn < 2; ++sgn) {
                Perturb& q = sgn == 0 ? plus : minus;
                Material mat = sc.materials[m];
                const float d = sgn == 0 ? hm : -hm;
                if (kind == 1) {
                    mat.base_color = Rgb(mat.base_color.r + d, mat.base_color.g + d, mat.base_color.b + d);
                } else {
                    const float alpha = mat.roughness * mat.roughness;
                    mat.roughness = std::sqrt(rmax(alpha + d, 0.0f));
                }
                q.kind = kind;
                q.index = m;
                q.outside = Bsdf::surface(mat, true);
                q.inside = Bsdf::surface(mat, false);
                if (kind == 1 && mat.absorption_mm > 0.0f) {
                    auto f = [&](float c) { return -fln(rclamp(c, 1.0e-4f, 1.0f)) / mat.absorption_mm; };
                    q.sigma = Rgb(f(mat.base_color.r), f(mat.base_color.g), f(mat.base_color.b));
                }
            }
            render(&plus, pa, pb, nullptr);
            render(&minus, ma, mb, nullptr);
            if (kind == 1) {
                for (int c = 0; c < 3; ++c) grads[4 * m + c] = delta(c) / (2.0 * (double)hm);
            } else {
                grads[4 * m + 3] = (delta(0) + delta(1) + delta(2)) / (2.0 * (double)hm);
            }
        }
    }
    for (uint32_t j = 0; j < nl; ++j) {
        const float power = sc.lights[j].power;
        grads[4 * nm + j] = 0.0;
        if (!(power > 0.0f)) continue;
        Perturb plus, minus;
        plus.kind = minus.kind = 3;
        plus.index = minus.index = j;
        plus.light_ratio = 1.0f + hm;
        minus.light_ratio = 1.0f - hm;
        render(&plus, pa, pb, nullptr);
        render(&minus, ma, mb, nullptr);
        const double dp = (double)power * (double)(plus.light_ratio - minus.light_ratio);
        grads[4 * nm + j] = (delta(0) + delta(1) + delta(2)) / dp;
    }
    return 0;
}

// Per-path radiance of explicit (pixel x, pixel y, sample) triples: out = r, g, b, alpha, rays.
// Every path is independent, so `threads` workers (0: the host's cores) give the same output.
void orc_paths(uint32_t h, const uint32_t* xys, uint32_t n, float* out5, uint32_t threads) {
    Loaded* l = get(h);
    if (!l) return;
    parallel_chunks(n, threads, [&](uint32_t b, uint32_t e, uint32_t) {
    for (uint32_t i = b; i < e; ++i) {
        PathStats st;
        Rgb c;
        float a;
        shade_pixel(l->scene, l->prep, xys[3 * i], xys[3 * i + 1], xys[3 * i + 2], c, a, st);
        out5[5 * i] = c.r; out5[5 * i + 1] = c.g; out5[5 * i + 2] = c.b; out5[5 * i + 3] = a; out5[5 * i + 4] = (float)st.rays;
    }
    });
}

// Nearest hits of a ray batch (ray = ox oy oz dx dy dz tmin tmax); hits = instance, triangle,
// t bits (0xffffffff instance: miss). `brute` uses every triangle instead of the BVH. stats2
// (may be null) gets inner-node visits and packet tests summed over the batch. `threads` workers
// (0: the host's cores) share the batch.
void orc_trace(uint32_t h, const float* rays, uint32_t n, uint32_t camera, uint32_t brute, uint32_t* hits, uint64_t* stats2,
               uint32_t threads) {
    Loaded* l = get(h);
    if (!l) return;
    std::mutex mu;
    uint64_t nodes = 0, packets = 0;
    parallel_chunks(n, threads, [&](uint32_t b, uint32_t e, uint32_t) {
    TraceStats st;
    for (uint32_t i = b; i < e; ++i) {
        const float* r = rays + 8 * i;
        Ray ray(Vec3(r[0], r[1], r[2]), Vec3(r[3], r[4], r[5]));
        ray.t_min = r[6];
        ray.t_max = r[7];
        RayHit hit;
        bool got = brute ? l->scene.geometry.trace_brute(ray, camera != 0, hit) : l->scene.geometry.trace(ray, camera != 0, hit, &st);
        hits[3 * i] = got ? hit.instance : 0xffffffffu;
        hits[3 * i + 1] = got ? hit.triangle : 0xffffffffu;
        hits[3 * i + 2] = got ? fbits(hit.t) : 0u;
    }
    std::lock_guard<std::mutex> lk(mu);
    nodes += st.nodes;
    packets += st.packets;
    });
    if (stats2) { stats2[0] = nodes; stats2[1] = packets; }
}
// Any-hit of a ray batch: occluded[i] = 1 when something lies in [tmin, tmax].
void orc_occluded(uint32_t h, const float* rays, uint32_t n, uint8_t* occluded) {
    Loaded* l = get(h);
    if (!l) return;
    for (uint32_t i = 0; i < n; ++i) {
        const float* r = rays + 8 * i;
        Ray ray(Vec3(r[0], r[1], r[2]), Vec3(r[3], r[4], r[5]));
        ray.t_min = r[6];
        ray.t_max = r[7];
        occluded[i] = l->scene.geometry.occluded(ray, false) ? 1 : 0;
    }
}

// The energy tables (u16 albedo[1024], schlick[1024], clear_in[17408], clear_out[17408];
// f32 albedo_avg[32], schlick_avg[32]).
void orc_energy_tables(uint16_t* u16s, float* f32s) {
    const EnergyTables& t = energy_tables();
    std::memcpy(u16s, t.albedo.data(), 1024 * 2);
    std::memcpy(u16s + 1024, t.schlick.data(), 1024 * 2);
    std::memcpy(u16s + 2048, t.clear_in.data(), 17408 * 2);
    std::memcpy(u16s + 2048 + 17408, t.clear_out.data(), 17408 * 2);
    std::memcpy(f32s, t.albedo_avg.data(), 32 * 4);
    std::memcpy(f32s + 32, t.schlick_avg.data(), 32 * 4);
}

// Known-answer helpers for the lights (light.rs tests): the number of selection entries and the
// static (by flux) probability of one; a light
// sample at x (Lights::sample: the selection at x, then sample_selected) into out10 = wi (3),
// distance, radiance (3), pdf, delta, shadow, 1 when there is one; the sky a camera ray sees
// along dir (Lights::escaped with no BSDF); the lights a ray (origin, dir, t_min, t_max) crosses,
// seen by the camera (bsdf_pdf < 0) or by a BSDF sample of that density from the ray's origin.
uint32_t orc_light_count(uint32_t h) {
    Loaded* l = get(h);
    return l ? (uint32_t)l->prep.lights.entries.size() : 0u;
}
float orc_light_flux_pmf(uint32_t h, uint32_t entry) {
    Loaded* l = get(h);
    if (!l || entry >= l->prep.lights.flux_pmf.size()) return 0.0f;
    return l->prep.lights.flux_pmf[entry];
}
uint32_t orc_light_sample(uint32_t h, const float* x3, float u_select, float u0, float u1, float* out10) {
    Loaded* l = get(h);
    if (!l) return 0;
    const Lights& L = l->prep.lights;
    LightSample s;
    if (!L.sample_selected(L.select(Vec3(x3[0], x3[1], x3[2])), u_select, u0, u1, s)) return 0;
    float v[10] = {s.wi.x, s.wi.y, s.wi.z, s.distance, s.radiance.r, s.radiance.g, s.radiance.b, s.pdf,
                   s.delta ? 1.0f : 0.0f, s.shadow ? 1.0f : 0.0f};
    std::memcpy(out10, v, sizeof v);
    return 1;
}
void orc_light_sky(uint32_t h, const float* dir3, float* out3) {
    Loaded* l = get(h);
    if (!l) return;
    Rgb e = l->prep.lights.escaped(Vec3(dir3[0], dir3[1], dir3[2]), nullptr, nullptr);
    out3[0] = e.r; out3[1] = e.g; out3[2] = e.b;
}
void orc_light_crossed(uint32_t h, const float* ray8, float bsdf_pdf, float* out3) {
    Loaded* l = get(h);
    if (!l) return;
    const Lights& L = l->prep.lights;
    Ray ray(Vec3(ray8[0], ray8[1], ray8[2]), Vec3(ray8[3], ray8[4], ray8[5]));
    ray.t_min = ray8[6];
    Selection at = L.select(ray.origin);
    Rgb c = L.crossed_from(ray, ray8[7], bsdf_pdf < 0.0f ? nullptr : &bsdf_pdf, &at, 0.0f);
    out3[0] = c.r; out3[1] = c.g; out3[2] = c.b;
}

// Known-answer helpers for the bitmaps (bitmap.rs, hdr.rs tests): decodes a BMAP payload; wh2 gets
// its decoded size; texels (3 w h floats, may be null) its pixels; then n bilinear lookups at
// uvw = (u, v, wrap) into out (3 floats each). 0 on success, 1 when it cannot be decoded (the
// reason in orc_error), 2 for a format outside this path.
uint32_t orc_bitmap(uint32_t format, uint32_t w, uint32_t h, const uint8_t* data, uint32_t len, uint32_t* wh2, float* texels,
                    uint32_t n, const float* uvw, float* out) {
    Image img;
    std::string reason;
    bool unsupported = false;
    if (!decode_bitmap(format, w, h, data, len, img, reason, unsupported)) {
        std::lock_guard<std::mutex> lk(g_mu);
        g_error = reason;
        return unsupported ? 2u : 1u;
    }
    wh2[0] = img.width;
    wh2[1] = img.height;
    if (texels)
        for (uint32_t y = 0; y < img.height; ++y)
            for (uint32_t x = 0; x < img.width; ++x) {
                Rgb c = img.texel(x, y);
                float* o = texels + 3 * ((size_t)y * img.width + x);
                o[0] = c.r; o[1] = c.g; o[2] = c.b;
            }
    for (uint32_t i = 0; i < n; ++i) {
        Rgb c = img.bilinear(uvw[3 * i], uvw[3 * i + 1], uvw[3 * i + 2] != 0.0f);
        out[3 * i] = c.r; out[3 * i + 1] = c.g; out[3 * i + 2] = c.b;
    }
    return 0;
}
// Distribution2D (bitmap.rs:330) over w x h weights: n samples at s (2 floats each) into out
// (u, v, pdf, pdf(u, v) per sample). 1 when the weights are all zero.
uint32_t orc_dist2d(uint32_t w, uint32_t h, const float* weights, uint32_t n, const float* s, float* out) {
    Distribution2D d;
    if (!Distribution2D::make(w, h, std::vector<float>(weights, weights + (size_t)w * h), d)) return 1;
    for (uint32_t i = 0; i < n; ++i) {
        float u, v, p;
        d.sample(s[2 * i], s[2 * i + 1], u, v, p);
        out[4 * i] = u; out[4 * i + 1] = v; out[4 * i + 2] = p; out[4 * i + 3] = d.pdf(u, v);
    }
    return 0;
}

// IES profiles (ies.rs tests): parses a file into out3 = peak, flux, symmetry (0 rotational,
// 1 quadrant, 2 bilateral 0-180, 3 bilateral 90-270, 4 full); 0 on success, 1 with the reason in
// orc_error. Then n intensities at (gamma, phi) degree pairs, and n shares of the peak towards
// local unit directions (3 floats each).
uint32_t orc_ies(const uint8_t* bytes, uint32_t len, float* out3, uint32_t n, const float* gamma_phi, float* intensities,
                 uint32_t m, const float* dirs, float* shapes) {
    IesProfile p;
    std::string reason;
    if (!IesProfile::parse(bytes, len, p, reason)) {
        std::lock_guard<std::mutex> lk(g_mu);
        g_error = reason;
        return 1;
    }
    out3[0] = p.peak;
    out3[1] = p.flux;
    out3[2] = (float)p.symmetry;
    for (uint32_t i = 0; i < n; ++i) intensities[i] = p.intensity(gamma_phi[2 * i], gamma_phi[2 * i + 1]);
    for (uint32_t i = 0; i < m; ++i) shapes[i] = p.shape(Vec3(dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]));
    return 0;
}

// The pixel filters (pixel_filter.rs:103): where n uniform numbers put a sample on one axis; and
// the Blackman-Harris table itself (256 floats).
void orc_filter_offset(uint32_t filter, const float* u, uint32_t n, float* out) {
    for (uint32_t i = 0; i < n; ++i) out[i] = filter_offset(filter, u[i]);
}
void orc_blackman_harris_table(float* out256) { std::memcpy(out256, blackman_harris_table(), 256 * sizeof(float)); }
// The edge mask of a scene (one byte per pixel; all zero without edge samples).
void orc_edge_mask(uint32_t h, uint8_t* out) {
    Loaded* l = get(h);
    if (!l) return;
    size_t n = (size_t)l->scene.render.width * l->scene.render.height;
    if (l->edges.empty()) std::memset(out, 0, n);
    else std::memcpy(out, l->edges.data(), n);
}

// Known-answer helpers: Pcg32, mix64, Sobol points, owen-scrambled sampler values, fmath.
void orc_pcg32(uint64_t seed, uint64_t stream, uint32_t n, uint32_t* out) {
    Pcg32 r = Pcg32::seeded(seed, stream);
    for (uint32_t i = 0; i < n; ++i) out[i] = r.next_u32();
}
uint64_t orc_mix64(uint64_t z) { return mix64(z); }
uint32_t orc_sobol(uint32_t dim, uint32_t index) { return sobol(dim, index); }
float orc_sampler_get1(uint32_t seed, uint32_t x, uint32_t y, uint32_t index, uint32_t dim) {
    return PixelSampler(seed, x, y, index).get1(dim);
}
void orc_fmath(uint32_t which, const float* in, uint32_t n, float* out) {
    for (uint32_t i = 0; i < n; ++i) {
        float x = in[i];
        switch (which) {
            case 0: out[i] = fsin(x); break;
            case 1: out[i] = fcos(x); break;
            case 2: out[i] = exp2(x); break;
            case 3: out[i] = log2(x); break;
            case 4: out[i] = fatan(x); break;
            case 5: out[i] = facos(x); break;
            default: out[i] = 0.0f;
        }
    }
}

}  // extern "C"
