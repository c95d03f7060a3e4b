// torch_rcs.cpp -- libtorch extension: the monostatic RCS of a sweep as a
// torch::autograd::Function of the mesh vertices and the frequencies, registered as
// the operator torch.ops.sagittasbr.rcs.
//
// Forward builds a scene from the current vertices (sbr_scene_create) and runs the
// sweep (sbr_run); sigma = 4 pi |S|^2 per (angle, frequency) sample
// (src/app/sweep.cu:228-230).  Backward turns dLoss/dsigma = w into the cotangent of
// every sample's field, g = 8 pi w S (dLoss = sum Re(conj(g) dS)), and calls
// sbr_adjoint, which re-traces the rays and differentiates along the frozen hit
// paths; it returns dLoss/dvertices and, summed over angles, dLoss/dfrequency.
// libtorch only carries tensors: all tracing runs in libsbr through its C ABI.

#include <torch/autograd.h>
#include <torch/library.h>
#include <torch/torch.h>

#include <cmath>
#include <memory>
#include <vector>

#include "sbr.h"

namespace {

void check(sbr_status s, const char* what) {
    TORCH_CHECK(s == SBR_OK, what, " failed: ", sbr_status_str(s), " (", sbr_last_error(), ")");
}

struct SceneOwner {
    sbr_scene* s = nullptr;
    ~SceneOwner() {
        if (s) sbr_scene_destroy(s);
    }
};

// Host copies of the sweep's inputs, kept alive for the job's pointers.
struct Sweep {
    std::vector<double> theta, phi, freqs;
    sbr_job job{};
    std::shared_ptr<SceneOwner> scene;
    std::vector<double> field;  // [n_angles * n_freqs * 2]
    int64_t nverts = 0;
    int32_t precision = SBR_PREC_MIXED;
};

std::vector<double> host_f64(const torch::Tensor& t) {
    auto c = t.detach().to(torch::kCPU, torch::kFloat64).contiguous().view({-1});
    return std::vector<double>(c.data_ptr<double>(), c.data_ptr<double>() + c.numel());
}

class RcsFunction : public torch::autograd::Function<RcsFunction> {
   public:
    static torch::Tensor forward(torch::autograd::AutogradContext* ctx, const torch::Tensor& verts,
                                 const torch::Tensor& freqs, const torch::Tensor& tris, const torch::Tensor& theta,
                                 const torch::Tensor& phi, int64_t nx, int64_t ny, double grid, int64_t max_bounces,
                                 double reflection_const, int64_t precision) {
        TORCH_CHECK(verts.dim() == 2 && verts.size(1) == 3, "verts must be [V, 3]");
        TORCH_CHECK(tris.dim() == 2 && tris.size(1) == 3, "tris must be [T, 3]");
        TORCH_CHECK(theta.numel() == phi.numel(), "theta and phi differ in length");
        auto sw = std::make_shared<Sweep>();
        sw->theta = host_f64(theta);
        sw->phi = host_f64(phi);
        sw->freqs = host_f64(freqs);
        sw->precision = (int32_t)precision;
        auto v = verts.detach().to(torch::kCPU, torch::kFloat32).contiguous();
        auto t = tris.detach().to(torch::kCPU, torch::kInt64).contiguous();
        TORCH_CHECK(t.numel() == 0 || (t.min().item<int64_t>() >= 0 && t.max().item<int64_t>() < verts.size(0)),
                    "triangle index out of range");
        auto t32 = t.to(torch::kInt32).contiguous();
        sw->nverts = v.size(0);

        sbr_build_opts bo{};
        bo.model_scale = 1.0;
        bo.device = -1;
        bo.want_fp64 = precision == SBR_PREC_FP64 ? 1 : 0;
        sw->scene = std::make_shared<SceneOwner>();
        check(sbr_scene_create(v.data_ptr<float>(), (size_t)v.size(0),
                               reinterpret_cast<const uint32_t*>(t32.data_ptr<int32_t>()), (size_t)t32.size(0), &bo,
                               &sw->scene->s),
              "sbr_scene_create");

        sbr_job& J = sw->job;
        J.theta_deg = sw->theta.data();
        J.phi_deg = sw->phi.data();
        J.n_angles = (int64_t)sw->theta.size();
        J.freq_hz = sw->freqs.data();
        J.n_freqs = (int64_t)sw->freqs.size();
        J.nx = (int32_t)nx;
        J.ny = (int32_t)ny;
        J.grid_size = grid;
        J.max_bounces = (int32_t)max_bounces;
        J.reflection_const = reflection_const;

        const int64_t n = J.n_angles * J.n_freqs;
        sw->field.assign((size_t)(2 * n), 0.0);
        std::vector<double> sigma((size_t)n);
        sbr_result res{};
        res.field = sw->field.data();
        res.sigma_m2 = sigma.data();
        sbr_run_opts ro{};
        ro.mode = SBR_MODE_BATCHED;
        ro.precision = (int32_t)precision;
        check(sbr_run(sw->scene->s, &J, 1, &res, &ro), "sbr_run");

        ctx->saved_data["sweep"] = c10::IValue(c10::make_intrusive<SweepHolder>(sw));
        ctx->saved_data["vdtype"] = (int64_t)verts.scalar_type();
        ctx->saved_data["fdtype"] = (int64_t)freqs.scalar_type();
        ctx->saved_data["vdev"] = verts.device().str();
        ctx->saved_data["fdev"] = freqs.device().str();
        auto out = torch::from_blob(sigma.data(), {J.n_angles, J.n_freqs}, torch::kFloat64).clone();
        return out.to(verts.device());
    }

    static torch::autograd::variable_list backward(torch::autograd::AutogradContext* ctx,
                                                   torch::autograd::variable_list grad_out) {
        auto sw = ctx->saved_data["sweep"].toCustomClass<SweepHolder>()->sweep;
        const sbr_job& J = sw->job;
        const int64_t n = J.n_angles * J.n_freqs;
        auto w = grad_out[0].detach().to(torch::kCPU, torch::kFloat64).contiguous().view({-1});
        TORCH_CHECK(w.numel() == n, "gradient of sigma has the wrong size");
        const double* wp = w.data_ptr<double>();
        std::vector<double> cot((size_t)(2 * n));
        for (int64_t s = 0; s < n; ++s) {
            cot[2 * s] = 8.0 * M_PI * wp[s] * sw->field[2 * s];
            cot[2 * s + 1] = 8.0 * M_PI * wp[s] * sw->field[2 * s + 1];
        }
        std::vector<double> gx((size_t)(3 * sw->nverts)), gf((size_t)n);
        sbr_run_opts ro{};
        ro.mode = SBR_MODE_BATCHED;
        ro.precision = sw->precision;
        check(sbr_adjoint(sw->scene->s, &J, 1, &ro, cot.data(), gx.data(), gf.data()), "sbr_adjoint");
        sw->scene.reset();

        const auto vdtype = (c10::ScalarType)ctx->saved_data["vdtype"].toInt();
        const auto fdtype = (c10::ScalarType)ctx->saved_data["fdtype"].toInt();
        const torch::Device vdev(ctx->saved_data["vdev"].toStringRef());
        const torch::Device fdev(ctx->saved_data["fdev"].toStringRef());
        // clone: the blobs are local vectors, and .to() returns its input unchanged when
        // device and dtype already match
        auto gverts = torch::from_blob(gx.data(), {sw->nverts, 3}, torch::kFloat64).clone().to(vdev, vdtype);
        auto gfreq = torch::from_blob(gf.data(), {J.n_angles, J.n_freqs}, torch::kFloat64).sum(0).to(fdev, fdtype);
        torch::autograd::variable_list g(11);
        g[0] = gverts;
        g[1] = gfreq;
        return g;
    }

    // Carries the sweep (scene handle, host inputs, fields) from forward to backward.
    struct SweepHolder : torch::CustomClassHolder {
        explicit SweepHolder(std::shared_ptr<Sweep> s) : sweep(std::move(s)) {}
        std::shared_ptr<Sweep> sweep;
    };
};

torch::Tensor rcs(const torch::Tensor& verts, const torch::Tensor& freqs, const torch::Tensor& tris,
                  const torch::Tensor& theta, const torch::Tensor& phi, int64_t nx, int64_t ny, double grid,
                  int64_t max_bounces, double reflection_const, int64_t precision) {
    return RcsFunction::apply(verts, freqs, tris, theta, phi, nx, ny, grid, max_bounces, reflection_const, precision);
}

}  // namespace

TORCH_LIBRARY(sagittasbr, m) {
    m.class_<RcsFunction::SweepHolder>("_SweepHolder");
    m.def("rcs(Tensor verts, Tensor freqs, Tensor tris, Tensor theta, Tensor phi, int nx, int ny, float grid, "
          "int max_bounces, float reflection_const=1.0, int precision=0) -> Tensor",
          &rcs);
}
