// plan.cpp -- sbr_plan: launcher frames, aperture clipping, the work-item table
// and the device result buffers; execute / results / run.
//
// The per-angle launcher frame restates src/app/sweep.cu:342-364
//   dir = (sin t cos p, sin t sin p, cos t), rayDir = -dir,
//   up = (0,1,0) or (1,0,0) when |dir.y| > 0.99,
//   U = unit(up x dir) G, V = unit(dir x U) G, llc = 10 G dir - U/2 - V/2,
// and k / ray area restate src/app/sweep.cu:50-53.  Two things are added:
//  * aperture clipping: rays whose (s, t) launcher coordinates fall outside the
//    projection of the scene's bounding box cannot hit anything (their hit count
//    stays 0 and they add nothing to the PO sum), so only the clipped rectangle of
//    pixels (plus a one-pixel margin) is launched;
//  * in SBR_PREC_MIXED the launch plane is moved from 10 G to just outside the
//    scene along dir and the distance moved is added back to the FP64 path, which
//    keeps FP32 ray coordinates small.  The first-hit tMin test is unchanged
//    because no geometry lies between the two planes.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "plan.hpp"

using namespace sbr;

namespace {

template <class R>
struct Fr {
    R dir[3], u[3], v[3], llc[3];
};

template <class R>
Fr<R> frame(double thetaDeg, double phiDeg, R G) {
    const R pi = R(M_PI);
    R th = R(thetaDeg) * pi / R(180.0);
    R ph = R(phiDeg) * pi / R(180.0);
    Fr<R> f;
    f.dir[0] = std::sin(th) * std::cos(ph);
    f.dir[1] = std::sin(th) * std::sin(ph);
    f.dir[2] = std::cos(th);
    R up[3] = {R(0), R(1), R(0)};
    if (std::fabs(f.dir[1]) > R(0.99)) { up[0] = R(1); up[1] = R(0); }
    auto crs = [](const R* a, const R* b, R* o) {
        o[0] = a[1] * b[2] - a[2] * b[1];
        o[1] = -(a[0] * b[2] - a[2] * b[0]);
        o[2] = a[0] * b[1] - a[1] * b[0];
    };
    auto unitScale = [](R* a, R G) {
        R l = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
        for (int k = 0; k < 3; ++k) a[k] = (a[k] / l) * G;
    };
    crs(up, f.dir, f.u);
    unitScale(f.u, G);
    crs(f.dir, f.u, f.v);
    unitScale(f.v, G);
    for (int k = 0; k < 3; ++k) f.llc[k] = (R(10.0) * G) * f.dir[k] - R(0.5) * f.u[k] - R(0.5) * f.v[k];
    return f;
}

template <class T>
sbr_status upload(T** d, const std::vector<T>& h, int64_t& bytes) {
    size_t n = std::max<size_t>(h.size(), 1) * sizeof(T);
    cudaError_t e = cudaMalloc(d, n);
    if (e != cudaSuccess) return fail(SBR_ERR_OOM, "plan allocation failed");
    bytes += (int64_t)n;
    if (!h.empty()) SBR_CUDA(cudaMemcpy(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    return SBR_OK;
}

template <class T>
sbr_status dalloc(T** d, size_t count, int64_t& bytes) {
    size_t n = std::max<size_t>(count, 1) * sizeof(T);
    cudaError_t e = cudaMalloc(d, n);
    if (e != cudaSuccess) return fail(SBR_ERR_OOM, "plan allocation failed");
    bytes += (int64_t)n;
    return SBR_OK;
}
// Zeroed on the plan's stream, so the plan's first launches come after the zeros
// (a cudaMemset on the legacy stream is not ordered with a non-blocking stream).
template <class T>
sbr_status zalloc(T** d, size_t count, int64_t& bytes, cudaStream_t st) {
    sbr_status r = dalloc(d, count, bytes);
    if (r != SBR_OK) return r;
    SBR_CUDA(cudaMemsetAsync(*d, 0, std::max<size_t>(count, 1) * sizeof(T), st));
    return SBR_OK;
}

void release(sbr_plan* p) {
    if (!p) return;
    sbr::DeviceGuard device_guard;
    cudaSetDevice(p->scene->device);
    if (p->stream) cudaStreamSynchronize(p->stream);
    if (p->graph) cudaGraphExecDestroy(p->graph);
    cudaFree(p->d_segs);
    cudaFree(p->d_seg_base);
    cudaFree(p->d_jobs);
    cudaFree(p->d_freqs);
    cudaFree(p->d_quantum);
    cudaFree(p->d_acc);
    cudaFree(p->d_acc_stats);
    cudaFree(p->d_field);
    cudaFree(p->d_stats);
    cudaFree(p->d_queue);
    cudaFree(p->d_zbuf);
    cudaFree(p->d_tile_cnt);
    cudaFree(p->d_tile_list);
    cudaFree(p->d_segpol);
    cudaFree(p->d_scenes);
    if (p->ev0) cudaEventDestroy(p->ev0);
    if (p->ev1) cudaEventDestroy(p->ev1);
    delete p;
}

sbr_status check_device_errors(sbr_plan* p) {
    uint32_t e = 0;
    SBR_CUDA(cudaMemcpy(&e, p->d_err, sizeof(e), cudaMemcpyDeviceToHost));
    if (e) clear_device_word(p->d_err);
    if (e & DEV_ERR_CANCEL) return fail(SBR_ERR_CANCELLED, "run cancelled");
    if (e & DEV_ERR_BUDGET) return fail(SBR_ERR_TIMEOUT, "traversal iteration budget exceeded");
    if (e & DEV_ERR_STACK) return fail(SBR_ERR_STACK, "traversal stack overflow");
    return SBR_OK;
}

}  // namespace

namespace sbr {

sbr_status validate_run(const sbr_scene* s, const sbr_job* jobs, size_t n_jobs, const sbr_run_opts& o) {
    if (!s || (!jobs && n_jobs)) return fail(SBR_ERR_INVALID_ARG, "null scene or jobs");
    if (o.mode != SBR_MODE_BATCHED && o.mode != SBR_MODE_PER_ANGLE) return fail(SBR_ERR_INVALID_ARG, "bad mode");
    if (o.precision < SBR_PREC_MIXED || o.precision > SBR_PREC_FP64) return fail(SBR_ERR_INVALID_ARG, "bad precision");
    if (o.polarization != SBR_POL_SCALAR && o.polarization != SBR_POL_HHVV)
        return fail(SBR_ERR_INVALID_ARG, "bad polarization");
    const bool pol = o.polarization == SBR_POL_HHVV;
    if (pol && o.precision == SBR_PREC_FP32)
        return fail(SBR_ERR_UNSUPPORTED, "polarisation tracking runs in SBR_PREC_MIXED or SBR_PREC_FP64");
    if (o.tile_cap < 0 || o.tile_cap > 1024) return fail(SBR_ERR_INVALID_ARG, "tile_cap outside 0..1024");
    for (size_t j = 0; j < n_jobs; ++j) {
        const sbr_job& J = jobs[j];
        if (J.n_angles < 0 || (J.n_angles > 0 && (!J.theta_deg || !J.phi_deg)))
            return fail(SBR_ERR_INVALID_ARG, "job angles");
        if (J.n_freqs < 1 || !J.freq_hz) return fail(SBR_ERR_INVALID_ARG, "job needs at least one frequency");
        if (J.n_freqs > max_freqs_per_job()) return fail(SBR_ERR_TOO_LARGE, "more than 128 frequencies in one job");
        if (pol && 2 * J.n_freqs > max_freqs_per_job())
            return fail(SBR_ERR_TOO_LARGE, "more than 64 frequencies in one polarised job");
        if (J.nx <= 0 || J.ny <= 0) return fail(SBR_ERR_INVALID_ARG, "n_x and n_y must be positive");
        if ((int64_t)J.nx * (int64_t)J.ny > (int64_t(1) << 31) - 1)
            return fail(SBR_ERR_TOO_LARGE, "more than 2^31-1 rays per angle");
        if (J.max_bounces < 0) return fail(SBR_ERR_INVALID_ARG, "max_bounces < 0");
        if (!(J.grid_size > 0) || !std::isfinite(J.grid_size)) return fail(SBR_ERR_INVALID_ARG, "grid_size");
        if (!std::isfinite(J.reflection_const)) return fail(SBR_ERR_NONFINITE, "reflection_const");
        for (int64_t a = 0; a < J.n_angles; ++a)
            if (!std::isfinite(J.theta_deg[a]) || !std::isfinite(J.phi_deg[a]))
                return fail(SBR_ERR_NONFINITE, "non-finite angle");
        for (int64_t f = 0; f < J.n_freqs; ++f)
            if (!(J.freq_hz[f] > 0) || !std::isfinite(J.freq_hz[f])) return fail(SBR_ERR_INVALID_ARG, "frequency");
    }
    return SBR_OK;
}

sbr_status build_tables(const sbr_scene* const* scenes, const int32_t* job_scene, const sbr_job* jobs,
                        size_t n_jobs, const sbr_run_opts& o, TableSink& sink, TableTotals& tot) {
    const double c0 = 299792458.0;
    tot = TableTotals{};
    int64_t item = 0, sample = 0;
    int32_t nfreq = 0;
    for (size_t j = 0; j < n_jobs; ++j) {
        const sbr_job& J = jobs[j];
        const int32_t si = job_scene ? job_scene[j] : 0;
        const sbr_scene* s = scenes[si];
        const double* lo = s->aabb_lo;
        const double* hi = s->aabb_hi;
        const double diag = std::sqrt((hi[0] - lo[0]) * (hi[0] - lo[0]) + (hi[1] - lo[1]) * (hi[1] - lo[1]) +
                                      (hi[2] - lo[2]) * (hi[2] - lo[2]));
        JobConst jc{};
        jc.scene = si;
        jc.nx = J.nx;
        jc.ny = J.ny;
        jc.n_freqs = (int32_t)J.n_freqs;
        jc.max_bounces = J.max_bounces;
        jc.freq_base = nfreq;
        jc.inv_nx = 1.0 / double(J.nx);
        jc.inv_ny = 1.0 / double(J.ny);
        jc.refl = J.reflection_const;
        jc.reflf = float(J.reflection_const);
        if (!sink.job(jc)) return fail(SBR_ERR_TOO_LARGE, "table capacity exceeded (jobs)");
        tot.k_max = std::max<int>(tot.k_max, (int)J.n_freqs);
        // k and the PO scale (src/app/sweep.cu:50-53); FP32 copies in FP32 arithmetic
        const double G = J.grid_size;
        const double area = (G * G) / double(int64_t(J.nx) * int64_t(J.ny));
        const float Gf = float(G);
        const float areaf = (Gf * Gf) / float(int64_t(J.nx) * int64_t(J.ny));
        double rmax = std::pow(std::max(1.0, std::fabs(J.reflection_const)), double(J.max_bounces));
        double quantum[128];
        for (int64_t f = 0; f < J.n_freqs; ++f) {
            FreqConst fc{};
            double lambda = c0 / J.freq_hz[f];
            fc.k = 2.0 * M_PI / lambda;
            fc.scale = fc.k * area / (4.0 * M_PI);
            fc.turns = fc.k / M_PI;
            fc.turns_hi = float(fc.turns);
            fc.turns_lo = float(fc.turns - double(fc.turns_hi));
            float lambdaf = 299792458.0f / float(J.freq_hz[f]);
            fc.kf = 2.0f * float(M_PI) / lambdaf;
            fc.scalef = fc.kf * areaf / (4.0f * float(M_PI));
            // |field| <= rays * k A/(4 pi) * 2 * max(1,R)^maxB; 2^60 units cover it with margin
            double bound = double(int64_t(J.nx) * int64_t(J.ny)) * std::max(fc.scale, double(fc.scalef)) * 2.0 * rmax;
            double q = bound / 1152921504606846976.0;  // 2^60
            if (!std::isfinite(q) || !(q > 0))
                return fail(SBR_ERR_TOO_LARGE, "field bound overflows (reflection_const^max_bounces too large)");
            fc.quantum = q;
            fc.inv_quantum = 1.0 / q;
            if (!sink.freq(fc)) return fail(SBR_ERR_TOO_LARGE, "table capacity exceeded (frequencies)");
            quantum[f] = q;
            ++nfreq;
        }
        for (int64_t a = 0; a < J.n_angles; ++a) {
            Segment g{};
            Fr<double> fd = frame<double>(J.theta_deg[a], J.phi_deg[a], G);
            Fr<float> ff = frame<float>(J.theta_deg[a], J.phi_deg[a], Gf);
            // clipped pixel rectangle: projection of the 8 box corners on (U, V)
            double smin = INFINITY, smax = -INFINITY, tmin = INFINITY, tmax = -INFINITY, pmax = -INFINITY;
            double uu = fd.u[0] * fd.u[0] + fd.u[1] * fd.u[1] + fd.u[2] * fd.u[2];
            double vv = fd.v[0] * fd.v[0] + fd.v[1] * fd.v[1] + fd.v[2] * fd.v[2];
            for (int c = 0; c < 8; ++c) {
                double P[3] = {(c & 1) ? hi[0] : lo[0], (c & 2) ? hi[1] : lo[1], (c & 4) ? hi[2] : lo[2]};
                double r[3] = {P[0] - fd.llc[0], P[1] - fd.llc[1], P[2] - fd.llc[2]};
                double sc = (r[0] * fd.u[0] + r[1] * fd.u[1] + r[2] * fd.u[2]) / uu;
                double tc = (r[0] * fd.v[0] + r[1] * fd.v[1] + r[2] * fd.v[2]) / vv;
                smin = std::min(smin, sc); smax = std::max(smax, sc);
                tmin = std::min(tmin, tc); tmax = std::max(tmax, tc);
                pmax = std::max(pmax, P[0] * fd.dir[0] + P[1] * fd.dir[1] + P[2] * fd.dir[2]);
            }
            auto clampi = [](double x, int n) { return (int)std::min<double>(std::max<double>(x, -1.0), double(n)); };
            int i0 = clampi(std::ceil(smin * J.nx - 0.5) - 1, J.nx), i1 = clampi(std::floor(smax * J.nx - 0.5) + 1, J.nx);
            int j0 = clampi(std::ceil(tmin * J.ny - 0.5) - 1, J.ny), j1 = clampi(std::floor(tmax * J.ny - 0.5) + 1, J.ny);
            i0 = std::max(i0, 0); j0 = std::max(j0, 0);
            i1 = std::min(i1, J.nx - 1); j1 = std::min(j1, J.ny - 1);
            g.i0 = i0;
            g.j0 = j0;
            g.ni = std::max(0, i1 - i0 + 1);
            g.nj = std::max(0, j1 - j0 + 1);
            if (J.max_bounces == 0) g.ni = g.nj = 0;
            double shift = 0.0;
            if (o.precision == SBR_PREC_MIXED) {
                shift = 10.0 * G - pmax - (0.01 + 1e-3 * diag);
                if (!(shift > 0)) shift = 0.0;
            }
            for (int k = 0; k < 3; ++k) {
                g.dir[k] = fd.dir[k];
                g.u[k] = fd.u[k];
                g.v[k] = fd.v[k];
                g.llc[k] = fd.llc[k] - shift * fd.dir[k];
                if (o.precision == SBR_PREC_FP32) {
                    g.llcf[k] = ff.llc[k];
                    g.uf[k] = ff.u[k];
                    g.vf[k] = ff.v[k];
                    g.rdf[k] = -ff.dir[k];
                } else {
                    g.llcf[k] = float(g.llc[k]);
                    g.uf[k] = float(fd.u[k]);
                    g.vf[k] = float(fd.v[k]);
                    g.rdf[k] = float(-fd.dir[k]);
                }
            }
            g.shift = shift;
            // pixel coordinates on the launcher: s(P) = (P - llc).U / |U|^2 * nx - 1/2
            for (int k = 0; k < 3; ++k) {
                g.ps[k] = fd.u[k] / uu * J.nx;
                g.pt[k] = fd.v[k] / vv * J.ny;
            }
            g.ps[3] = -(fd.llc[0] * g.ps[0] + fd.llc[1] * g.ps[1] + fd.llc[2] * g.ps[2]) - 0.5;
            g.pt[3] = -(fd.llc[0] * g.pt[0] + fd.llc[1] * g.pt[1] + fd.llc[2] * g.pt[2]) - 0.5;
            g.zbase = 0;
            g.job = (int32_t)j;
            g.angle = (int32_t)a;
            int bx = (g.ni + kBlockW - 1) / kBlockW, by = (g.nj + kBlockH - 1) / kBlockH;
            g.blocks_x = bx;
            g.blocks = bx * by;
            // up to 8 blocks (256 rays) per warp item in batched mode, fewer when a
            // segment is small; one block per item in per-angle mode, where a single
            // segment must spread over the whole GPU
            int bpi = o.mode == SBR_MODE_BATCHED ? std::max(1, std::min(8, g.blocks / 1024)) : 1;
            if (o.blocks_per_item > 0) bpi = std::min(o.blocks_per_item, 1024);
            g.blocks_per_item = bpi;
            g.item_base = item;
            g.sample_base = sample;
            item += (g.blocks + bpi - 1) / bpi;
            sample += J.n_freqs;
            tot.n_rays_clipped += (int64_t)g.ni * g.nj;
            tot.n_rays_grid += (int64_t)J.nx * J.ny;
            if (!sink.segment(g, item, quantum, (int)J.n_freqs))
                return fail(SBR_ERR_TOO_LARGE, "table capacity exceeded (angles or samples)");
            tot.n_segs += 1;
        }
    }
    tot.n_items = item;
    tot.n_samples = sample;
    if (tot.n_segs > INT32_MAX) return fail(SBR_ERR_TOO_LARGE, "too many angles");
    return SBR_OK;
}

}  // namespace sbr

namespace {

// Collects the tables of a plan in its host vectors.
struct PlanSink : sbr::TableSink {
    sbr_plan* p;
    explicit PlanSink(sbr_plan* pl) : p(pl) { p->seg_base.push_back(0); }
    bool job(const JobConst& j) override { p->jobs.push_back(j); return true; }
    bool freq(const FreqConst& f) override { p->freqs.push_back(f); return true; }
    bool segment(const Segment& g, int64_t next_item, const double* q, int nf) override {
        p->segs.push_back(g);
        p->seg_base.push_back(next_item);
        for (int f = 0; f < nf; ++f) p->quantum.push_back(q[f]);
        return true;
    }
};

}  // namespace

namespace {

sbr_status plan_create(sbr_scene* const* scenes, size_t n_scenes, const int32_t* job_scene, const sbr_job* jobs,
                       size_t n_jobs, const sbr_run_opts* opts, sbr_plan** out);

// Autotuner of batched plans: every candidate (blocks per work item, persistent
// CTAs per SM) -- the automatic setting among them -- runs a sample of the plan
// (up to 128 angles spread evenly over the jobs' angle lists) twice, the second
// run timed on the device, and the fastest setting is written into `o`.
sbr_status autotune(sbr_scene* const* scenes, size_t n_scenes, const int32_t* job_scene, const sbr_job* jobs,
                    size_t n_jobs, sbr_run_opts& o) {
    const int64_t per_job = std::max<int64_t>(2, 128 / (int64_t)std::max<size_t>(1, n_jobs));
    std::vector<std::vector<double>> th(n_jobs), ph(n_jobs);
    std::vector<sbr_job> sj(jobs, jobs + n_jobs);
    for (size_t j = 0; j < n_jobs; ++j) {
        const int64_t na = jobs[j].n_angles, m = std::min(na, per_job);
        for (int64_t q = 0; q < m; ++q) {
            const int64_t a = m > 1 ? (q * (na - 1)) / (m - 1) : 0;
            th[j].push_back(jobs[j].theta_deg[a]);
            ph[j].push_back(jobs[j].phi_deg[a]);
        }
        sj[j].theta_deg = th[j].data();
        sj[j].phi_deg = ph[j].data();
        sj[j].n_angles = m;
    }
    const int bpis[] = {0, 1, 2, 4, 8, 16};
    const int ctas[] = {0, 6};
    // both tree widths when a single-scene plan's scene holds an 8-wide tree
    std::vector<int> widths{o.node_width};
    if (!job_scene && o.node_width == 0 && scenes[0]->d_nodes8) widths = {4, 8};
    double best = INFINITY;
    int best_bpi = 0, best_ctas = 0, best_w = o.node_width;
    for (int w : widths)
    for (int c : ctas) {
        for (int b : bpis) {
            sbr_run_opts t = o;
            t.autotune = 0;
            t.use_graph = 0;
            t.blocks_per_item = b;
            t.ctas_per_sm = c;
            t.node_width = w;
            sbr_plan* pl = nullptr;
            sbr_status st = plan_create(scenes, n_scenes, job_scene, sj.data(), n_jobs, &t, &pl);
            if (st != SBR_OK) return st;
            sbr_result r{};
            for (int rep = 0; rep < 2 && st == SBR_OK; ++rep) {
                st = sbr_plan_execute(pl);
                if (st == SBR_OK) st = sbr_plan_results(pl, &r);
            }
            sbr_plan_destroy(pl);
            if (st != SBR_OK) return st;
            if (r.device_ms < best) {
                best = r.device_ms;
                best_bpi = b;
                best_ctas = c;
                best_w = w;
            }
        }
    }
    o.blocks_per_item = best_bpi;
    o.ctas_per_sm = best_ctas;
    o.node_width = best_w;
    return SBR_OK;
}

// Plan over one scene (job_scene null) or several scenes on one device.
sbr_status plan_create(sbr_scene* const* scenes, size_t n_scenes, const int32_t* job_scene, const sbr_job* jobs,
                       size_t n_jobs, const sbr_run_opts* opts, sbr_plan** out) {
    if (!out) return fail(SBR_ERR_INVALID_ARG, "out is null");
    *out = nullptr;
    if (!scenes || n_scenes == 0) return fail(SBR_ERR_INVALID_ARG, "no scene");
    sbr_run_opts o{};
    if (opts) o = *opts;
    sbr_scene* s = scenes[0];
    sbr_status vs = validate_run(s, jobs, n_jobs, o);
    if (vs != SBR_OK) return vs;
    if (o.blocks_per_item < 0 || o.ctas_per_sm < 0) return fail(SBR_ERR_INVALID_ARG, "negative tuning option");
    if (o.node_width != 0 && o.node_width != 4 && o.node_width != 8)
        return fail(SBR_ERR_INVALID_ARG, "node_width must be 0, 4 or 8");
    if (o.first_hit < SBR_FIRST_HIT_AUTO || o.first_hit > SBR_FIRST_HIT_TRAVERSE)
        return fail(SBR_ERR_INVALID_ARG, "first_hit must be SBR_FIRST_HIT_AUTO, _RASTER or _TRAVERSE");
    if (o.node_width == 8 && !s->d_nodes8)
        return fail(SBR_ERR_UNSUPPORTED, "node_width 8 needs a scene built with sbr_build_opts.node_width = 8");
    for (size_t k = 0; k < n_scenes; ++k) {
        if (!scenes[k]) return fail(SBR_ERR_INVALID_ARG, "null scene");
        if (scenes[k]->device != s->device) return fail(SBR_ERR_INVALID_ARG, "scenes of one plan share a device");
    }
    if (job_scene)
        for (size_t j = 0; j < n_jobs; ++j)
            if (job_scene[j] < 0 || (size_t)job_scene[j] >= n_scenes)
                return fail(SBR_ERR_INVALID_ARG, "job scene index out of range");
    sbr::DeviceGuard device_guard;
    SBR_CUDA(cudaSetDevice(s->device));
    if (o.precision == SBR_PREC_FP64) {
        for (size_t k = 0; k < n_scenes; ++k) {
            sbr_status st = ensure_fp64(scenes[k]);
            if (st != SBR_OK) return st;
        }
    }

    if (o.autotune && o.mode == SBR_MODE_BATCHED && n_jobs > 0) {
        sbr_status st = autotune(scenes, n_scenes, job_scene, jobs, n_jobs, o);
        if (st != SBR_OK) return st;
    }

    sbr_plan* p = new sbr_plan();
    p->scene = s;
    p->blocks_per_item = o.blocks_per_item;
    p->multi = job_scene != nullptr;
    if (p->multi)
        for (size_t k = 0; k < n_scenes; ++k) p->scene_views.push_back(scenes[k]->view());
    p->mode = o.mode;
    p->prec = o.precision;
    p->pol = o.polarization;
    p->use_graph = o.use_graph;
    p->ctas_per_sm = o.ctas_per_sm;
    p->num_sms = s->num_sms;
    p->stream = o.stream ? (cudaStream_t)o.stream : s->stream;
    p->scene_view = s->view();
    p->node_width = !job_scene && ((o.node_width == 0 && s->d_nodes8) || o.node_width == 8) ? 8 : 4;
    if (p->node_width == 4) p->scene_view.nodes8 = nullptr;  // the sweep kernel walks the 4-wide tree
    p->d_err = s->d_err;
    p->d_cancel = s->d_cancel;

    PlanSink sink(p);
    TableTotals tot;
    const sbr_scene* const* cs = scenes;
    sbr_status bs = build_tables(cs, job_scene, jobs, n_jobs, o, sink, tot);
    if (bs != SBR_OK) {
        release(p);
        return bs;
    }
    p->k_max = tot.k_max;
    p->n_segs = tot.n_segs;
    p->n_items = tot.n_items;
    p->n_samples = tot.n_samples;
    p->n_rays_clipped = tot.n_rays_clipped;
    p->n_rays_grid = tot.n_rays_grid;
    p->n_pol = p->pol == SBR_POL_HHVV ? 2 : 1;
    if (p->n_pol == 2) {
        // per angle: HH / VV unit vectors and the reference launch plane; the
        // accumulator units are per (sample, polarisation)
        p->segpol.resize(p->segs.size());
        for (size_t g = 0; g < p->segs.size(); ++g) {
            const Segment& G = p->segs[g];
            const double th = jobs[G.job].theta_deg[G.angle] * M_PI / 180.0;
            const double ph = jobs[G.job].phi_deg[G.angle] * M_PI / 180.0;
            SegPol& q = p->segpol[g];
            q.eh[0] = -std::sin(ph); q.eh[1] = std::cos(ph); q.eh[2] = 0.0;
            q.ev[0] = std::cos(th) * std::cos(ph); q.ev[1] = std::cos(th) * std::sin(ph); q.ev[2] = -std::sin(th);
            q.plane = G.dir[0] * G.llc[0] + G.dir[1] * G.llc[1] + G.dir[2] * G.llc[2] + G.shift;
            q.pad = 0.0;
        }
        std::vector<double> qp(2 * p->quantum.size());
        for (size_t s = 0; s < p->quantum.size(); ++s) qp[2 * s] = qp[2 * s + 1] = p->quantum[s];
        p->quantum.swap(qp);
    }

    // first-hit rasterisation (batched mixed-precision single-scene plans): asked
    // for, or, by default, where the plan launches at least 8 rays per triangle per
    // angle (binning costs per triangle and angle, the walk it replaces per ray:
    // measured on B200, the 2.15 M-triangle aircraft at 18 rays per triangle gains
    // 8 %, the 200k-triangle ellipsoid at 0.4 loses 23 %)
    int64_t live_segs = 0;
    for (const auto& g : p->segs) live_segs += g.blocks > 0;
    const bool dense = (double)p->n_rays_clipped >= 8.0 * (double)s->ntris * (double)std::max<int64_t>(live_segs, 1);
    p->raster = o.mode == SBR_MODE_BATCHED && o.precision == SBR_PREC_MIXED && p->n_items > 0 && !p->multi &&
                (o.first_hit == SBR_FIRST_HIT_RASTER || (o.first_hit == SBR_FIRST_HIT_AUTO && dense));
    if (p->raster) {
        // per tile: 32 first-hit entries (8 B), a count and `cap` list entries (4 B);
        // a chunk holds at most 8 GiB of them (or one segment)
        p->tile_cap = o.tile_cap > 0 ? (uint32_t)o.tile_cap : 48u;
        const int64_t budget = (int64_t(8) << 30) / (32 * 8 + 4 + 4 * (int64_t)p->tile_cap);
        sbr_plan::Chunk c{0, 0, 0, 0, 0, 0};
        for (size_t g = 0; g < p->segs.size(); ++g) {
            const int64_t tiles = p->segs[g].blocks;
            // (the binning launch's grid.y is the chunk's segment count: at most 65535)
            if (c.seg_end > c.seg_begin && (c.tiles + tiles > budget || c.seg_end - c.seg_begin >= 65535)) {
                c.item_end = p->seg_base[c.seg_end];
                p->chunks.push_back(c);
                c = sbr_plan::Chunk{c.seg_end, c.seg_end, p->seg_base[c.seg_end], 0, 0, 0};
            }
            p->segs[g].tbase = (int32_t)c.tiles;
            p->segs[g].zbase = 32 * c.tiles;
            c.tiles += tiles;
            c.zcount = 32 * c.tiles;
            c.seg_end = (int64_t)g + 1;
        }
        c.item_end = p->seg_base[c.seg_end];
        p->chunks.push_back(c);
        for (const auto& ch : p->chunks) {
            p->zbuf_elems = std::max(p->zbuf_elems, ch.zcount);
            p->tiles_max = std::max(p->tiles_max, ch.tiles);
        }
    }

    sbr_status st;
    int64_t& b = p->device_bytes;
    if (p->raster) {
        // every entry of a chunk is written by its tile raster before the trace reads it
        const int64_t b0 = b;
        if ((st = dalloc(&p->d_zbuf, (size_t)p->zbuf_elems, b)) != SBR_OK ||
            (st = dalloc(&p->d_tile_cnt, (size_t)p->tiles_max, b)) != SBR_OK ||
            (st = dalloc(&p->d_tile_list, (size_t)p->tiles_max * p->tile_cap, b)) != SBR_OK) {
            if (o.first_hit == SBR_FIRST_HIT_RASTER) {
                release(p);
                return st;
            }
            // chosen automatically: without room for its buffers the plan walks instead
            // (a failed cudaMalloc is not sticky; its error is cleared here)
            cudaGetLastError();
            cudaFree(p->d_zbuf);
            cudaFree(p->d_tile_cnt);
            cudaFree(p->d_tile_list);
            p->d_zbuf = nullptr;
            p->d_tile_cnt = nullptr;
            p->d_tile_list = nullptr;
            b = b0;
            p->raster = false;
            p->chunks.clear();
            p->zbuf_elems = 0;
            p->tiles_max = 0;
            st = SBR_OK;
        }
    }
    if ((st = upload(&p->d_segs, p->segs, b)) != SBR_OK || (st = upload(&p->d_seg_base, p->seg_base, b)) != SBR_OK ||
        (st = upload(&p->d_jobs, p->jobs, b)) != SBR_OK || (st = upload(&p->d_freqs, p->freqs, b)) != SBR_OK ||
        (st = upload(&p->d_quantum, p->quantum, b)) != SBR_OK ||
        (p->n_pol == 2 && (st = upload(&p->d_segpol, p->segpol, b)) != SBR_OK) ||
        (p->multi && (st = upload(&p->d_scenes, p->scene_views, b)) != SBR_OK) ||
        (st = zalloc(&p->d_acc, 2 * (size_t)p->n_samples * p->n_pol * kAccReplicas, b, p->stream)) != SBR_OK ||
        (st = zalloc(&p->d_acc_stats, 4 * (size_t)p->n_segs, b, p->stream)) != SBR_OK ||
        (st = zalloc(&p->d_field, 2 * (size_t)p->n_samples * p->n_pol, b, p->stream)) != SBR_OK ||
        (st = zalloc(&p->d_stats, 4 * (size_t)p->n_segs, b, p->stream)) != SBR_OK ||
        (st = zalloc(&p->d_queue, 1 + (size_t)p->n_samples + p->chunks.size(), b, p->stream)) != SBR_OK) {
        release(p);
        return st;
    }
    cudaError_t e;
    if ((e = cudaEventCreate(&p->ev0)) != cudaSuccess || (e = cudaEventCreate(&p->ev1)) != cudaSuccess) {
        release(p);
        return cuda_fail(e, "cudaEventCreate");
    }
    *out = p;
    return SBR_OK;
}

}  // namespace

extern "C" {

sbr_status sbr_plan_create(sbr_scene* s, const sbr_job* jobs, size_t n_jobs, const sbr_run_opts* opts,
                           sbr_plan** out) {
    return plan_create(&s, 1, nullptr, jobs, n_jobs, opts, out);
}

sbr_status sbr_plan_create_multi(sbr_scene* const* scenes, size_t n_scenes, const int32_t* job_scene,
                                 const sbr_job* jobs, size_t n_jobs, const sbr_run_opts* opts, sbr_plan** out) {
    if (!job_scene && n_jobs) return fail(SBR_ERR_INVALID_ARG, "job_scene is required");
    return plan_create(scenes, n_scenes, job_scene, jobs, n_jobs, opts, out);
}

sbr_status sbr_plan_execute(sbr_plan* p) {
    if (!p) return fail(SBR_ERR_INVALID_ARG, "plan is null");
    sbr::DeviceGuard device_guard;
    SBR_CUDA(cudaSetDevice(p->scene->device));
    SBR_CUDA(cudaEventRecord(p->ev0, p->stream));
    if (p->use_graph && p->mode == SBR_MODE_BATCHED) {
        if (!p->graph) {
            // size the persistent grid outside capture, then capture the launches
            cudaGraph_t g;
            SBR_CUDA(cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal));
            sbr_status st = plan_launch(p, false, nullptr);
            cudaError_t e = cudaStreamEndCapture(p->stream, &g);
            if (st != SBR_OK) return st;
            if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
            e = cudaGraphInstantiate(&p->graph, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
        }
        SBR_CUDA(cudaGraphLaunch(p->graph, p->stream));
    } else {
        sbr_status st = plan_launch(p, false, nullptr);
        if (st != SBR_OK) return st;
    }
    SBR_CUDA(cudaEventRecord(p->ev1, p->stream));
    p->executed = true;
    return SBR_OK;
}

sbr_status sbr_plan_results(sbr_plan* p, sbr_result* out) {
    if (!p || !out) return fail(SBR_ERR_INVALID_ARG, "null argument");
    if (!p->executed) return fail(SBR_ERR_INVALID_ARG, "plan was not executed");
    sbr::DeviceGuard device_guard;
    SBR_CUDA(cudaSetDevice(p->scene->device));
    SBR_CUDA(cudaEventSynchronize(p->ev1));
    sbr_status st = check_device_errors(p);
    if (st != SBR_OK) return st;
    float ms = 0.0f;
    SBR_CUDA(cudaEventElapsedTime(&ms, p->ev0, p->ev1));
    out->device_ms = ms;
    const int64_t n_out = p->n_samples * p->n_pol;
    std::vector<double> f(2 * (size_t)n_out);
    if (n_out)
        SBR_CUDA(cudaMemcpyAsync(f.data(), p->d_field, f.size() * sizeof(double), cudaMemcpyDeviceToHost, p->stream));
    if (out->stats && p->n_segs)
        SBR_CUDA(cudaMemcpyAsync(out->stats, p->d_stats, 4 * (size_t)p->n_segs * sizeof(uint64_t),
                                 cudaMemcpyDeviceToHost, p->stream));
    SBR_CUDA(cudaStreamSynchronize(p->stream));
    for (int64_t i = 0; i < n_out; ++i) {
        double re = f[2 * i], im = f[2 * i + 1];
        if (out->field) { out->field[2 * i] = re; out->field[2 * i + 1] = im; }
        double sigma = 4.0 * M_PI * (re * re + im * im);
        if (out->sigma_m2) out->sigma_m2[i] = sigma;
        if (out->rcs_dbsm) out->rcs_dbsm[i] = 10.0 * std::log10(std::max(sigma, 1e-10));
    }
    return SBR_OK;
}

sbr_status sbr_plan_device_results(sbr_plan* p, const double** d_field, const uint64_t** d_stats) {
    if (!p) return fail(SBR_ERR_INVALID_ARG, "plan is null");
    if (d_field) *d_field = p->d_field;
    if (d_stats) *d_stats = reinterpret_cast<const uint64_t*>(p->d_stats);
    return SBR_OK;
}

sbr_status sbr_plan_info_get(const sbr_plan* p, sbr_plan_info* out) {
    if (!p || !out) return fail(SBR_ERR_INVALID_ARG, "null argument");
    out->n_samples = p->n_samples;
    out->n_job_angles = p->n_segs;
    out->n_items = p->n_items;
    out->n_rays_clipped = p->n_rays_clipped;
    out->n_rays_grid = p->n_rays_grid;
    out->n_pol = p->n_pol;
    out->blocks_per_item = p->blocks_per_item;
    out->ctas_per_sm = p->ctas_per_sm;
    out->node_width = p->node_width;
    out->first_hit = p->raster ? SBR_FIRST_HIT_RASTER : SBR_FIRST_HIT_TRAVERSE;
    int64_t launches = 1;
    if (p->mode == SBR_MODE_BATCHED && p->raster) {
        for (const auto& ch : p->chunks) launches += (ch.tiles > 0 ? 2 : 0) + (ch.item_end > ch.item_begin ? 1 : 0);
    } else if (p->mode == SBR_MODE_BATCHED) {
        launches += p->n_items > 0 ? 1 : 0;
    }
    else
        for (size_t g = 0; g < p->segs.size(); ++g)
            if (p->seg_base[g + 1] > p->seg_base[g]) launches += p->jobs[p->segs[g].job].n_freqs;
    out->launches_per_execute = (int32_t)std::min<int64_t>(launches, INT32_MAX);
    out->device_bytes = p->device_bytes;
    out->h2d_bytes = (int64_t)(p->segs.size() * sizeof(Segment) + p->seg_base.size() * sizeof(int64_t) +
                               p->jobs.size() * sizeof(JobConst) + p->freqs.size() * sizeof(FreqConst) +
                               p->quantum.size() * sizeof(double) + p->segpol.size() * sizeof(SegPol));
    out->d2h_bytes = (int64_t)(2 * p->n_samples * p->n_pol * sizeof(double) + 4 * p->n_segs * sizeof(uint64_t) +
                               sizeof(uint32_t));
    return SBR_OK;
}

sbr_status sbr_plan_destroy(sbr_plan* p) {
    if (!p) return fail(SBR_ERR_INVALID_ARG, "plan is null");
    release(p);
    return SBR_OK;
}

sbr_status sbr_run(sbr_scene* s, const sbr_job* jobs, size_t n_jobs, sbr_result* out, const sbr_run_opts* opts) {
    if (!out) return fail(SBR_ERR_INVALID_ARG, "out is null");
    sbr_plan* p = nullptr;
    sbr_status st = sbr_plan_create(s, jobs, n_jobs, opts, &p);
    if (st != SBR_OK) return st;
    st = sbr_plan_execute(p);
    if (st == SBR_OK) st = sbr_plan_results(p, out);
    release(p);
    return st;
}

sbr_status sbr_trace_records(sbr_scene* s, const sbr_job* job, const sbr_run_opts* opts, sbr_ray_record* out) {
    if (!s || !job || !out) return fail(SBR_ERR_INVALID_ARG, "null argument");
    sbr::DeviceGuard device_guard;
    SBR_CUDA(cudaSetDevice(s->device));
    // hit records do not depend on the polarisation: trace them with the scalar plan
    sbr_run_opts o{};
    if (opts) o = *opts;
    o.polarization = SBR_POL_SCALAR;
    sbr_plan* p = nullptr;
    sbr_status st = sbr_plan_create(s, job, 1, &o, &p);
    if (st != SBR_OK) return st;
    long long n = (long long)job->n_angles * job->nx * job->ny;
    sbr_ray_record* d = nullptr;
    cudaError_t e = cudaMalloc(&d, std::max<long long>(n, 1) * sizeof(sbr_ray_record));
    if (e != cudaSuccess) {
        release(p);
        return fail(SBR_ERR_OOM, "record buffer allocation failed");
    }
    st = fill_records(d, n, p->stream);
    if (st == SBR_OK) st = plan_launch(p, true, d);
    if (st == SBR_OK) {
        e = cudaStreamSynchronize(p->stream);
        if (e != cudaSuccess) st = cuda_fail(e, "trace records");
    }
    if (st == SBR_OK) st = check_device_errors(p);
    if (st == SBR_OK && n > 0) {
        e = cudaMemcpy(out, d, n * sizeof(sbr_ray_record), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) st = cuda_fail(e, "record copy");
    }
    cudaFree(d);
    release(p);
    return st;
}

sbr_status sbr_trace_ray_list(sbr_scene* s, const sbr_job* job, const sbr_run_opts* opts, const int32_t* rays,
                              size_t n_rays, sbr_ray_record* out) {
    if (!s || !job || (n_rays && (!rays || !out))) return fail(SBR_ERR_INVALID_ARG, "null argument");
    for (size_t k = 0; k < n_rays; ++k) {
        const int32_t a = rays[3 * k], i = rays[3 * k + 1], j = rays[3 * k + 2];
        if (a < 0 || a >= job->n_angles || i < 0 || i >= job->nx || j < 0 || j >= job->ny)
            return fail(SBR_ERR_INVALID_ARG, "listed ray outside the job's angles or ray grid");
    }
    sbr::DeviceGuard device_guard;
    SBR_CUDA(cudaSetDevice(s->device));
    sbr_run_opts o{};
    if (opts) o = *opts;
    o.polarization = SBR_POL_SCALAR;
    o.mode = SBR_MODE_BATCHED;
    o.first_hit = SBR_FIRST_HIT_TRAVERSE;
    sbr_plan* p = nullptr;
    sbr_status st = sbr_plan_create(s, job, 1, &o, &p);
    if (st != SBR_OK) return st;
    int32_t* d_rays = nullptr;
    sbr_ray_record* d = nullptr;
    const size_t n = std::max<size_t>(n_rays, 1);
    cudaError_t e = cudaMalloc(&d_rays, n * 3 * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMalloc(&d, n * sizeof(sbr_ray_record));
    if (e != cudaSuccess) st = fail(SBR_ERR_OOM, "ray list allocation failed");
    if (st == SBR_OK && n_rays) {
        e = cudaMemcpyAsync(d_rays, rays, n_rays * 3 * sizeof(int32_t), cudaMemcpyHostToDevice, p->stream);
        if (e != cudaSuccess) st = cuda_fail(e, "ray list copy");
    }
    if (st == SBR_OK) st = fill_records(d, (long long)n_rays, p->stream);
    if (st == SBR_OK) st = trace_list_launch(p, d_rays, (long long)n_rays, d);
    if (st == SBR_OK) {
        e = cudaStreamSynchronize(p->stream);
        if (e != cudaSuccess) st = cuda_fail(e, "trace ray list");
    }
    if (st == SBR_OK) st = check_device_errors(p);
    if (st == SBR_OK && n_rays) {
        e = cudaMemcpy(out, d, n_rays * sizeof(sbr_ray_record), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) st = cuda_fail(e, "record copy");
    }
    cudaFree(d);
    cudaFree(d_rays);
    release(p);
    return st;
}

}  // extern "C"
