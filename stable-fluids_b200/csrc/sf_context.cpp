// sf_context.cpp -- the C ABI of stable-fluids-3d.h / stable-fluids-b200.h:
// context creation and validation, device memory, the step graph, views.
//
// Reference behaviour followed (Xayah-Graphics/stable-fluids backend-cuda.cu):
//   create   :481-680  (validation 516-528/538-540, 1-based handles 544/551,
//                       allocation 560-581, initial values 583-606,
//                       one captured graph per step 608-675)
//   destroy  :682-690  update_* :692-719  step :721-726  get_view :728-800
// Differences, all additive: a null desc/context/out pointer, a non-positive
// grid size or cell size, or a negative iteration count is rejected with
// BACKEND_FAILURE instead of being dereferenced or used; destroy(nullptr) is a
// no-op; update_* accept host pointers too (cudaMemcpyDefault).

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <new>
#include <cstdio>
#include <string>
#include <string_view>
#include <utility>
#include <vector>

#include "sf_batch.h"
#include "sf_boundary.h"
#include "sf_launch.h"
#include "sf_types.h"
#include "sf_unet.h"
#include "stable-fluids-3d.h"
#include "stable-fluids-b200.h"

namespace sfb {
namespace {

struct Range {
    explicit Range(const char* name) { nvtxRangePushA(name); }
    ~Range() { nvtxRangePop(); }
    Range(const Range&) = delete;
    Range& operator=(const Range&) = delete;
};

struct ScalarField {
    StableFluidsScalarFieldDesc desc{};
    ScalarBC bc{};
    float* data = nullptr;    // BF16 elements in a BF16-storage context
    float* temp = nullptr;    // BF16 elements in a BF16-storage context
    float* source = nullptr;
    float* view = nullptr;    // BF16 storage: FP32 copy for views and updates
};

struct VectorField {
    StableFluidsVectorFieldDesc desc{};
    float* data[3] = {nullptr, nullptr, nullptr};
    // staged upload (stable_fluids_b200_stage_vector_field): the next values,
    // copied in on the caller's copy stream and moved into `data` by the next
    // step; `staged` says a copy is waiting
    float* stage[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t stage_ready = nullptr;  // the staged copy has landed (copy stream)
    cudaEvent_t stage_free = nullptr;   // the step has taken it (context stream)
    bool staged = false;
};

// Asynchronous read-back (stable_fluids_b200_read_view_async): the view's
// arrays are copied into `snap` on the context stream, then to the host on
// the caller's copy stream.
struct Snapshot {
    float* snap[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t taken = nullptr;  // the copies into snap are done (context stream)
    cudaEvent_t sent = nullptr;   // the copies to the host are done (copy stream)
    bool used = false;
};

struct Context {
    StableFluidsSimulationConfig config{};
    StableFluidsB200Options options{};
    cudaStream_t stream = nullptr;
    cudaStream_t body_stream = nullptr;  // captures the body of the residual-driven loop
    bool owns_stream = false;
    Dims dims{};
    size_t cells = 0;
    size_t field_bytes = 0;
    FlowBC flow{};

    void* slab = nullptr;
    size_t slab_bytes = 0;
    // Advected fields: FP32, or BF16 elements (bf16) behind the same
    // pointers; views of a BF16 context are FP32 copies made at get_view.
    bool bf16 = false;
    float* vel[3] = {nullptr, nullptr, nullptr};
    float* temp[3] = {nullptr, nullptr, nullptr};
    float* view_vel[3] = {nullptr, nullptr, nullptr};
    void* packed = nullptr;  // packed velocity: float4, or 4 x BF16
    float* pressure = nullptr;
    float* divergence = nullptr;
    float* magnitude = nullptr;
    float* scratch = nullptr;
    float* scratch2 = nullptr;  // red-black solves: the split right-hand side
    DeviceStats* stats = nullptr;
    DeviceStats* host_stats = nullptr;  // pinned
    // learned warm start: the network (not owned), the plain candidate and
    // its Jacobi scratch, and the plain candidate's residual sums
    net::Net* network = nullptr;
    float* alt = nullptr;
    float* alt_scratch = nullptr;
    DeviceStats* alt_stats = nullptr;
    // coarse-grid prediction: restricted divergence and previous pressure,
    // the network's coarse output (null: the network runs on the full grid)
    float* coarse_b = nullptr;
    float* coarse_p = nullptr;
    float* coarse_out = nullptr;
    Dims coarse_dims() const { return Dims{dims.nx / 2, dims.ny / 2, dims.nz / 2, 0}; }
    std::vector<ScalarField> scalars;
    std::vector<VectorField> vectors;

    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t ready = nullptr;
    bool residual_enabled = false;
    int step_kernels = 0;  // kernel nodes in the step graph
    int check_kernels = 0;  // kernel nodes in the residual loop's body
    bool blocked = true;   // temporally blocked stencil passes

    Snapshot snapshot;

    ~Context() {
        for (auto& v : vectors) {
            for (auto* p : v.stage)
                if (p) cudaFree(p);
            if (v.stage_ready) cudaEventDestroy(v.stage_ready);
            if (v.stage_free) cudaEventDestroy(v.stage_free);
        }
        for (auto* p : snapshot.snap)
            if (p) cudaFree(p);
        if (snapshot.taken) cudaEventDestroy(snapshot.taken);
        if (snapshot.sent) cudaEventDestroy(snapshot.sent);
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (ready) cudaEventDestroy(ready);
        if (slab) cudaFree(slab);
        if (host_stats) cudaFreeHost(host_stats);
        if (body_stream) cudaStreamDestroy(body_stream);
        if (owns_stream && stream) cudaStreamDestroy(stream);
    }
};

bool valid_scalar_type(uint32_t t) { return t <= STABLE_FLUIDS_SCALAR_BOUNDARY_PERIODIC; }

// backend-cuda.cu:521-525
bool validate_scalar(const StableFluidsScalarBoundaryConfig& b) {
    const StableFluidsScalarBoundaryFaceDesc* f = &b.x_minus;
    for (int a = 0; a < 3; ++a) {
        const auto lo = f[2 * a].type, hi = f[2 * a + 1].type;
        if (!valid_scalar_type(lo) || !valid_scalar_type(hi)) return false;
        if ((lo == STABLE_FLUIDS_SCALAR_BOUNDARY_PERIODIC) != (hi == STABLE_FLUIDS_SCALAR_BOUNDARY_PERIODIC)) return false;
    }
    return true;
}

ScalarBC flatten(const StableFluidsScalarBoundaryConfig& b) {
    ScalarBC o{};
    const StableFluidsScalarBoundaryFaceDesc* f = &b.x_minus;
    for (int k = 0; k < 6; ++k) {
        o.type[k] = static_cast<int32_t>(f[k].type);
        o.value[k] = f[k].value;
    }
    for (int a = 0; a < 3; ++a) o.periodic[a] = f[2 * a].type == STABLE_FLUIDS_SCALAR_BOUNDARY_PERIODIC && f[2 * a + 1].type == STABLE_FLUIDS_SCALAR_BOUNDARY_PERIODIC;
    return o;
}

bool env_flag(const char* name) {
    const char* v = std::getenv(name);
    return v != nullptr && *v != '\0' && std::string_view(v) != "0";
}

void apply_env_overrides(StableFluidsB200Options& o) {
    if (const char* v = std::getenv("STABLE_FLUIDS_B200_SCHEME")) {
        const std::string_view s(v);
        if (s == "jacobi" || s == "JACOBI" || s == "1") o.scheme = STABLE_FLUIDS_B200_SCHEME_JACOBI;
        else if (s == "rbgs" || s == "RBGS" || s == "0") o.scheme = STABLE_FLUIDS_B200_SCHEME_RBGS;
    }
    if (const char* v = std::getenv("STABLE_FLUIDS_B200_ITERATIONS_PER_PASS")) o.iterations_per_pass = std::atoi(v);
    if (const char* v = std::getenv("STABLE_FLUIDS_B200_RESIDUAL_TOLERANCE")) o.residual_tolerance = static_cast<float>(std::atof(v));
    if (const char* v = std::getenv("STABLE_FLUIDS_B200_MAX_PRESSURE_ITERATIONS")) o.max_pressure_iterations = std::atoi(v);
    if (const char* v = std::getenv("STABLE_FLUIDS_B200_WARM_START")) {
        const std::string_view s(v);
        if (s == "previous" || s == "1") o.warm_start = STABLE_FLUIDS_B200_WARM_START_PREVIOUS;
        else if (s == "zero" || s == "0") o.warm_start = STABLE_FLUIDS_B200_WARM_START_ZERO;
        else if (s == "learned" || s == "2") o.warm_start = STABLE_FLUIDS_B200_WARM_START_LEARNED;
    }
    if (env_flag("STABLE_FLUIDS_B200_COMPUTE_RESIDUAL")) o.compute_residual = 1;
    if (env_flag("STABLE_FLUIDS_B200_WARM_START_COARSEN")) o.warm_start_coarsening = 1;
    if (const char* v = std::getenv("STABLE_FLUIDS_B200_STORAGE")) {
        const std::string_view s(v);
        if (s == "bf16" || s == "BF16" || s == "1") o.storage = STABLE_FLUIDS_B200_STORAGE_BF16;
        else if (s == "fp32" || s == "FP32" || s == "0") o.storage = STABLE_FLUIDS_B200_STORAGE_FP32;
    }
}

void default_options(StableFluidsB200Options& o) {
    o = StableFluidsB200Options{};
    o.scheme = STABLE_FLUIDS_B200_SCHEME_RBGS;
    o.warm_start = STABLE_FLUIDS_B200_WARM_START_ZERO;
    o.iterations_per_pass = 0;
    o.residual_tolerance = 0.0f;
    o.max_pressure_iterations = 0;
    o.residual_check_interval = 8;
    o.compute_residual = 0;
    o.warm_start_trial_iterations = 8;
}

bool validate_options(const StableFluidsB200Options& o) {
    if (o.scheme > STABLE_FLUIDS_B200_SCHEME_JACOBI) return false;
    if (o.warm_start > STABLE_FLUIDS_B200_WARM_START_LEARNED) return false;
    if (o.warm_start_trial_iterations < 0) return false;
    if (o.storage > STABLE_FLUIDS_B200_STORAGE_BF16) return false;
    if (o.iterations_per_pass < 0) return false;
    if (!(o.residual_tolerance >= 0.0f) || !std::isfinite(o.residual_tolerance)) return false;
    if (o.residual_tolerance > 0.0f && (o.max_pressure_iterations <= 0 || o.residual_check_interval <= 0)) return false;
    return true;
}

// Carves every device array out of one allocation, each 256-byte aligned.
struct SlabPlan {
    struct Item {
        void** where;
        size_t bytes;
    };
    std::vector<Item> items;
    void add(void** where, size_t bytes) { items.push_back({where, bytes}); }
    size_t total() const {
        size_t t = 0;
        for (const auto& it : items) t += (it.bytes + 255) & ~static_cast<size_t>(255);
        return t;
    }
    void assign(void* base) const {
        auto* p = static_cast<char*>(base);
        for (const auto& it : items) {
            *it.where = p;
            p += (it.bytes + 255) & ~static_cast<size_t>(255);
        }
    }
};

// ---- stages of the step, in the reference's order (backend-cuda.cu:612-671).
// Each enqueues its work on the context stream (inside the step-graph capture
// or, for profiling, directly) and adds its kernel count to `launches`.
struct Stages {
    Context& c;
    int launches = 0;
    cudaError_t e = cudaSuccess;

    bool ok(cudaError_t r, int kernels = 1) {
        if (r == cudaSuccess) launches += kernels;
        else if (e == cudaSuccess) e = r;
        return r == cudaSuccess;
    }
    float h() const { return c.config.cell_size; }
    float alpha_v() const { return c.config.dt * c.config.viscosity / (h() * h()); }  // :622
    float alpha_s(const ScalarField& f) const { return c.config.dt * f.desc.diffusion / (h() * h()); }  // :656
    bool any_scalar_advects() const {
        for (const auto& f : c.scalars)
            if (alpha_s(f) > 0.0f) return true;
        return false;
    }

    // 1. v += dt f field by field (:612-615), fused with packing the velocity
    //    for the advection gathers.
    void forces() {
        std::vector<const VectorField*> list;
        for (const auto& v : c.vectors)
            if (v.desc.usage == STABLE_FLUIDS_VECTOR_FIELD_FORCE) list.push_back(&v);
        const bool advect = alpha_v() > 0.0f;
        size_t k = 0;
        do {
            ForceArgs fa{};
            for (int comp = 0; comp < 3; ++comp) fa.vel[comp] = c.vel[comp];
            fa.dt = c.config.dt;
            fa.bf16 = c.bf16 ? 1 : 0;
            fa.n = c.cells;
            for (; k < list.size() && fa.force_count < kMaxForcesPerLaunch; ++k, ++fa.force_count)
                for (int comp = 0; comp < 3; ++comp) fa.force[fa.force_count][comp] = list[k]->data[comp];
            const bool last = k >= list.size();
            // Only the last launch packs; the SoA velocity is written when more
            // launches follow or when no advection reads the packed copy.
            fa.write_soa = (!last || !advect) ? 1 : 0;
            fa.packed = (last && advect) ? c.packed : nullptr;
            if (fa.force_count > 0 || fa.packed) ok(launch_force_pack(fa, c.stream));
        } while (k < list.size());
    }

    // 2. advection (:617-619); skipped when alpha <= 0 because the reference
    //    then never copies the advected velocity back (:623).
    void advect_velocity() {
        if (alpha_v() > 0.0f) ok(launch_advect_velocity(c.packed, c.temp[0], c.temp[1], c.temp[2], c.config.dt, c.dims, h(), c.flow, c.bf16, c.stream));
    }

    StencilArgs stencil(int kind, int init, int iterations, float coef, float* x, const float* b) {
        StencilArgs a{};
        a.kind = kind;
        a.scheme = static_cast<int>(c.options.scheme);
        a.init = init;
        a.iterations = iterations;
        a.per_pass = c.options.iterations_per_pass;
        a.coef = coef;
        a.out_scale = 1.0f;
        a.x = x;
        a.b = b;
        a.scratch = c.scratch;
        a.scratch2 = c.scratch2;
        a.dims = c.dims;
        a.flow = c.flow;
        a.launches = &launches;
        a.blocked = c.blocked ? 1 : 0;
        a.error_flag = &c.stats->error;
        a.bf16 = (c.bf16 && kind != KIND_PRESSURE) ? 1 : 0;
        return a;
    }

    // 3. implicit viscosity, x0 = advected velocity (:621-641).
    void diffuse_velocity() {
        if (!(alpha_v() > 0.0f)) return;
        for (int comp = 0; comp < 3; ++comp) ok(launch_stencil(stencil(KIND_VEL_X + comp, INIT_FROM_B, c.config.diffuse_iterations, alpha_v(), c.vel[comp], c.temp[comp]), c.stream), 0);
    }

    // 4. divergence (:643).
    void divergence() { ok(launch_divergence(c.divergence, c.vel[0], c.vel[1], c.vel[2], c.dims, h(), c.flow, c.bf16, c.stream)); }

    // 5. pressure from zero (:644-649), from the previous step's pressure, or
    //    from the learned warm start.
    void pressure() {
        const int init = c.options.warm_start == STABLE_FLUIDS_B200_WARM_START_ZERO ? INIT_ZERO : INIT_FROM_X;
        const bool residual_driven = c.options.residual_tolerance > 0.0f && capturing();
        int done = 0;  // iterations already run on the start that was kept
        if (c.options.warm_start == STABLE_FLUIDS_B200_WARM_START_LEARNED && c.network != nullptr) done = learned_start(residual_driven);
        if (residual_driven) {
            pressure_until_converged(init, done);
            return;
        }
        const int left = c.config.pressure_iterations - done;
        if (left > 0) ok(launch_stencil(stencil(KIND_PRESSURE, init, left, h() * h(), c.pressure, c.divergence), c.stream), 0);
    }

    // Learned warm start: the network predicts a start from (div, previous
    // pressure) in place; the previous pressure is kept as the plain
    // candidate. Both get the trial sweeps, both residuals are measured, and
    // the one with the smaller residual stays in c.pressure (its sums in
    // c.stats, the decision in used_fallback). Returns the sweeps run.
    int learned_start(bool residual_driven) {
        int trial = c.options.warm_start_trial_iterations;
        if (!residual_driven) trial = std::min(trial, c.config.pressure_iterations);
        ok(cudaMemcpyAsync(c.alt, c.pressure, c.field_bytes, cudaMemcpyDeviceToDevice, c.stream), 0);
        int predicted = 0;
        if (c.coarse_b != nullptr) {
            // the network on the 2x coarser grid (cell size 2h), its correction prolonged
            const float h2c = (2.0f * h()) * (2.0f * h());
            ok(launch_restrict2(c.divergence, c.coarse_b, c.dims, c.stream));
            ok(launch_restrict2(c.pressure, c.coarse_p, c.dims, c.stream));
            if (ok(net::predict(c.network, c.coarse_b, h2c, c.coarse_p, c.coarse_out, c.coarse_dims(), c.stream, &predicted, &c), 0)) launches += predicted;
            ok(launch_prolong_add(c.coarse_out, c.coarse_p, c.pressure, c.dims, c.stream));
        } else if (ok(net::predict(c.network, c.divergence, h() * h(), c.pressure, c.pressure, c.dims, c.stream, &predicted, &c), 0)) {
            launches += predicted;
        }
        if (trial > 0) {
            ok(launch_stencil(stencil(KIND_PRESSURE, INIT_FROM_X, trial, h() * h(), c.pressure, c.divergence), c.stream), 0);
            auto a = stencil(KIND_PRESSURE, INIT_FROM_X, trial, h() * h(), c.alt, c.divergence);
            a.scratch = c.alt_scratch;
            ok(launch_stencil(a, c.stream), 0);
        }
        ok(cudaMemsetAsync(c.stats, 0, offsetof(DeviceStats, rel_residual), c.stream), 0);
        ok(cudaMemsetAsync(c.alt_stats, 0, offsetof(DeviceStats, rel_residual), c.stream), 0);
        ok(launch_residual_sums(c.pressure, c.divergence, c.dims, h() * h(), c.flow, c.stats, c.stream));
        ok(launch_residual_sums(c.alt, c.divergence, c.dims, h() * h(), c.flow, c.alt_stats, c.stream));
        ok(launch_warm_start_select(c.stats, c.alt_stats, c.dims, c.flow.any_outflow ? 0 : 1, c.pressure, c.alt, c.stream), 2);
        return trial;
    }

    bool capturing() const {
        cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
        return cudaStreamIsCapturing(c.stream, &st) == cudaSuccess && st == cudaStreamCaptureStatusActive;
    }

    // Residual-driven solve: measure rel_res of the initial pressure, then a
    // WHILE graph node repeats {check_interval iterations, FP64 residual} while
    // rel_res > tolerance and fewer than max_pressure_iterations have run
    // (the count is rounded up to a multiple of the interval).
    // `done` iterations have run already (learned warm start), with the sums
    // of the current pressure in c.stats.
    void pressure_until_converged(int init, int done) {
        const int interval = c.options.residual_check_interval;
        const int max_it = ((c.options.max_pressure_iterations + interval - 1) / interval) * interval;
        const int singular = c.flow.any_outflow ? 0 : 1;
        const double tol = static_cast<double>(c.options.residual_tolerance);
        if (done == 0) {
            if (init == INIT_ZERO) ok(cudaMemsetAsync(c.pressure, 0, c.field_bytes, c.stream), 0);
            ok(cudaMemsetAsync(c.stats, 0, offsetof(DeviceStats, rel_residual), c.stream), 0);
            ok(launch_residual_sums(c.pressure, c.divergence, c.dims, h() * h(), c.flow, c.stats, c.stream));
        }
        cudaStreamCaptureStatus st;
        cudaGraph_t graph = nullptr;
        const cudaGraphNode_t* deps = nullptr;
        size_t ndeps = 0;
        cudaGraphConditionalHandle handle{};
        if (!ok(cudaStreamGetCaptureInfo(c.stream, &st, nullptr, &graph, &deps, &ndeps), 0)) return;
        if (!ok(cudaGraphConditionalHandleCreate(&handle, graph, 0, 0), 0)) return;
        ok(launch_residual_check(c.stats, c.dims, singular, 1, done, tol, max_it, handle, c.stream));
        if (!ok(cudaStreamGetCaptureInfo(c.stream, &st, nullptr, &graph, &deps, &ndeps), 0)) return;
        cudaGraphNodeParams cp{};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = handle;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node = nullptr;
        if (!ok(cudaGraphAddNode(&node, graph, deps, ndeps, &cp), 0)) return;
        if (!ok(cudaStreamUpdateCaptureDependencies(c.stream, &node, 1, cudaStreamSetCaptureDependencies), 0)) return;
        // the body, captured on the second stream
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        if (!ok(cudaStreamBeginCaptureToGraph(c.body_stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal), 0)) return;
        const cudaStream_t main = c.stream;
        c.stream = c.body_stream;
        const int before = launches;
        // Jacobi: the interval's last sweep also measures the residual of its
        // input (no separate pass); otherwise sweeps, then the residual pass
        if (!launch_pressure_interval_fused(stencil(KIND_PRESSURE, INIT_FROM_X, interval, h() * h(), c.pressure, c.divergence), c.stats, c.stream)) {
            // the same measurement point as the fused form for Jacobi
            const bool jacobi = c.options.scheme == STABLE_FLUIDS_B200_SCHEME_JACOBI;
            const int before_last = jacobi ? interval - 1 : interval;
            if (before_last > 0) ok(launch_stencil(stencil(KIND_PRESSURE, INIT_FROM_X, before_last, h() * h(), c.pressure, c.divergence), c.stream), 0);
            ok(launch_residual_sums(c.pressure, c.divergence, c.dims, h() * h(), c.flow, c.stats, c.stream));
            if (jacobi) ok(launch_stencil(stencil(KIND_PRESSURE, INIT_FROM_X, 1, h() * h(), c.pressure, c.divergence), c.stream), 0);
        }
        ok(launch_residual_check(c.stats, c.dims, singular, 0, interval, tol, max_it, handle, c.stream));
        c.check_kernels = launches - before;
        c.stream = main;
        cudaGraph_t captured = nullptr;
        ok(cudaStreamEndCapture(c.body_stream, &captured), 0);
        residual_measured = true;
    }
    bool residual_measured = false;

    // 6. projection (:650) + the FP64 residual of the pressure solve.
    void project() {
        // the residual-driven solve has measured the residual already
        const bool measure = c.residual_enabled && !residual_measured;
        ok(launch_project(c.vel[0], c.vel[1], c.vel[2], any_scalar_advects() ? c.packed : nullptr, c.pressure, c.divergence, c.dims, h(), h() * h(), c.flow, nullptr, c.bf16, c.stream));
        if (measure) {
            // projection reads p and div without changing them: the residual
            // of the solve is measured after it, by one separate pass
            ok(cudaMemsetAsync(c.stats, 0, offsetof(DeviceStats, rel_residual), c.stream), 0);
            ok(launch_residual_sums(c.pressure, c.divergence, c.dims, h() * h(), c.flow, c.stats, c.stream));
            ok(launch_residual_finalize(c.stats, c.dims, c.flow.any_outflow ? 0 : 1, c.config.pressure_iterations, c.stream));
        }
    }

    // 7. scalars: source, advection by the projected velocity, diffusion,
    //    dissipation (:652-668).
    void scalars() {
        for (auto& f : c.scalars) {
            const float a_s = alpha_s(f);
            const float factor = f.desc.dissipation > 0.0f ? 1.0f / (1.0f + c.config.dt * f.desc.dissipation) : 1.0f;  // :665
            if (a_s > 0.0f) {
                ok(launch_scalar_source_advect(c.packed, f.data, f.source, f.temp, c.config.dt, c.dims, h(), c.flow, f.bc, c.bf16, c.stream));
                auto a = stencil(KIND_SCALAR, INIT_FROM_B, c.config.diffuse_iterations, a_s, f.data, f.temp);
                a.scalar = f.bc;
                a.out_scale = factor;
                ok(launch_stencil(a, c.stream), 0);
            } else {
                ok(launch_scalar_source(f.data, f.source, c.config.dt, c.cells, c.bf16, c.stream));
                if (f.desc.dissipation > 0.0f) ok(launch_scale(f.data, factor, c.cells, c.bf16, c.stream));
            }
        }
    }

    // 8. post-projection divergence and |u| (:670-671).
    void diagnostics() { ok(launch_post_diagnostics(c.divergence, c.magnitude, c.vel[0], c.vel[1], c.vel[2], c.dims, h(), c.flow, c.bf16, c.stream)); }

    cudaError_t whole_step() {
        forces();
        advect_velocity();
        diffuse_velocity();
        divergence();
        pressure();
        project();
        scalars();
        diagnostics();
        return e;
    }
};

// The whole step as one graph (:608-675), replacing any previous one.
// Thread-local capture so other host threads' CUDA calls are unaffected.
cudaError_t build_graph(Context& c) {
    Range range("stable.create_context.graph");
    if (c.exec) cudaGraphExecDestroy(c.exec);
    if (c.graph) cudaGraphDestroy(c.graph);
    c.exec = nullptr;
    c.graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    Stages st{c};
    const cudaError_t rec = st.whole_step();
    c.step_kernels = st.launches;
    cudaGraph_t g = nullptr;
    const cudaError_t end = cudaStreamEndCapture(c.stream, &g);
    c.graph = g;
    if (rec != cudaSuccess || end != cudaSuccess || g == nullptr) {
        cudaGetLastError();
        return rec != cudaSuccess ? rec : (end != cudaSuccess ? end : cudaErrorStreamCaptureInvalidated);
    }
    if ((e = cudaGraphInstantiate(&c.exec, c.graph, 0)) != cudaSuccess) {
        c.exec = nullptr;
        cudaGetLastError();
        return e;
    }
    return cudaSuccess;
}

StableFluidsResult create(const StableFluidsContextCreateDesc* desc, const StableFluidsB200Options* options_in, bool env, void** out_context, StableFluidsScalarFieldHandle* out_s, uint32_t cap_s, StableFluidsVectorFieldHandle* out_v, uint32_t cap_v) {
    Range range("stable.create_context");
    if (out_context == nullptr) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    *out_context = nullptr;
    if (desc == nullptr) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    const auto& cfg = desc->config;
    if (cfg.nx <= 0 || cfg.ny <= 0 || cfg.nz <= 0) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    if (!(cfg.cell_size > 0.0f) || !std::isfinite(cfg.cell_size) || !std::isfinite(cfg.dt) || !std::isfinite(cfg.viscosity)) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    if (cfg.diffuse_iterations < 0 || cfg.pressure_iterations < 0) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    if (desc->scalar_field_count > 0 && desc->scalar_fields == nullptr) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    if (desc->vector_field_count > 0 && desc->vector_fields == nullptr) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    FlowBC flow{};
    if (!flatten_flow(cfg.flow_boundary, flow)) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;  // backend-cuda.cu:516-520
    for (uint32_t i = 0; i < desc->scalar_field_count; ++i)
        if (!validate_scalar(desc->scalar_fields[i].boundary)) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;

    StableFluidsB200Options options{};
    if (options_in) options = *options_in;
    else default_options(options);
    if (env) apply_env_overrides(options);
    if (!validate_options(options)) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;

    std::unique_ptr<Context> c{new (std::nothrow) Context{}};
    if (!c) return STABLE_FLUIDS_RESULT_OUT_OF_MEMORY;
    c->config = cfg;
    c->options = options;
    c->dims = Dims{cfg.nx, cfg.ny, cfg.nz, 0};
    c->cells = static_cast<size_t>(cfg.nx) * static_cast<size_t>(cfg.ny) * static_cast<size_t>(cfg.nz);
    c->field_bytes = c->cells * sizeof(float);
    c->flow = flow;
    c->residual_enabled = options.compute_residual != 0 || options.residual_tolerance > 0.0f;
    // Temporally blocked passes when asked for (iterations_per_pass >= 1);
    // the default one-launch-per-colour kernels are faster on B200 today.
    c->bf16 = options.storage == STABLE_FLUIDS_B200_STORAGE_BF16;
    c->blocked = !c->bf16 && (options.iterations_per_pass > 0 || env_flag("STABLE_FLUIDS_B200_BLOCKED_STENCIL"));

    // Handles are 1-based indices (:544, :551).
    for (uint32_t i = 0; i < desc->scalar_field_count; ++i) {
        ScalarField f;
        f.desc = desc->scalar_fields[i];
        f.bc = flatten(f.desc.boundary);
        c->scalars.push_back(f);
        if (out_s != nullptr && i < cap_s) out_s[i] = i + 1u;
    }
    for (uint32_t i = 0; i < desc->vector_field_count; ++i) {
        VectorField f;
        f.desc = desc->vector_fields[i];
        c->vectors.push_back(f);
        if (out_v != nullptr && i < cap_v) out_v[i] = i + 1u;
    }

    if (desc->stream != nullptr) c->stream = static_cast<cudaStream_t>(desc->stream);
    else {
        if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
        c->owns_stream = true;
    }
    if (cudaStreamCreateWithFlags(&c->body_stream, cudaStreamNonBlocking) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;

    {
        Range alloc("stable.create_context.alloc");
        SlabPlan plan;
        const size_t fb = c->field_bytes;
        const size_t sb = c->bf16 ? c->cells * 2 : fb;  // an advected field
        for (int k = 0; k < 3; ++k) plan.add(reinterpret_cast<void**>(&c->vel[k]), sb);
        for (int k = 0; k < 3; ++k) plan.add(reinterpret_cast<void**>(&c->temp[k]), sb);
        if (c->bf16)
            for (int k = 0; k < 3; ++k) plan.add(reinterpret_cast<void**>(&c->view_vel[k]), fb);
        plan.add(&c->packed, c->cells * 4 * (c->bf16 ? 2 : sizeof(float)));
        plan.add(reinterpret_cast<void**>(&c->pressure), fb);
        plan.add(reinterpret_cast<void**>(&c->divergence), fb);
        plan.add(reinterpret_cast<void**>(&c->magnitude), fb);
        plan.add(reinterpret_cast<void**>(&c->scratch), fb);
        // red-black solves split the right-hand side by colour into a second buffer
        if (options.scheme == STABLE_FLUIDS_B200_SCHEME_RBGS) plan.add(reinterpret_cast<void**>(&c->scratch2), fb);
        plan.add(reinterpret_cast<void**>(&c->stats), sizeof(DeviceStats));
        if (options.warm_start == STABLE_FLUIDS_B200_WARM_START_LEARNED) {
            plan.add(reinterpret_cast<void**>(&c->alt), fb);
            plan.add(reinterpret_cast<void**>(&c->alt_scratch), fb);
            plan.add(reinterpret_cast<void**>(&c->alt_stats), sizeof(DeviceStats));
            if (options.warm_start_coarsening != 0 && c->dims.nx % 2 == 0 && c->dims.ny % 2 == 0 && c->dims.nz % 2 == 0) {
                const size_t cb = fb / 8;
                plan.add(reinterpret_cast<void**>(&c->coarse_b), cb);
                plan.add(reinterpret_cast<void**>(&c->coarse_p), cb);
                plan.add(reinterpret_cast<void**>(&c->coarse_out), cb);
            }
        }
        for (auto& f : c->scalars) {
            plan.add(reinterpret_cast<void**>(&f.data), sb);
            plan.add(reinterpret_cast<void**>(&f.temp), sb);
            if (c->bf16) plan.add(reinterpret_cast<void**>(&f.view), fb);
            plan.add(reinterpret_cast<void**>(&f.source), fb);
        }
        for (auto& f : c->vectors)
            for (int k = 0; k < 3; ++k) plan.add(reinterpret_cast<void**>(&f.data[k]), fb);
        // Host-side fault injection for the OUT_OF_MEMORY path (tests only).
        if (env_flag("STABLE_FLUIDS_B200_INJECT_ALLOC_FAILURE")) return STABLE_FLUIDS_RESULT_OUT_OF_MEMORY;
        c->slab_bytes = plan.total();
        if (cudaMalloc(&c->slab, c->slab_bytes) != cudaSuccess) {
            c->slab = nullptr;
            cudaGetLastError();
            return STABLE_FLUIDS_RESULT_OUT_OF_MEMORY;
        }
        plan.assign(c->slab);
        if (cudaMallocHost(reinterpret_cast<void**>(&c->host_stats), sizeof(DeviceStats)) != cudaSuccess) {
            c->host_stats = nullptr;
            cudaGetLastError();
            return STABLE_FLUIDS_RESULT_OUT_OF_MEMORY;
        }
        std::memset(c->host_stats, 0, sizeof(DeviceStats));
        if (cudaEventCreateWithFlags(&c->ready, cudaEventDisableTiming) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    }

    {
        // Initial values (:583-606): everything zero, then the non-zero
        // scalar and vector initial values.
        Range init("stable.create_context.init");
        if (cudaMemsetAsync(c->slab, 0, c->slab_bytes, c->stream) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
        for (auto& f : c->scalars) {
            if (f.desc.initial_value == 0.0f) continue;
            if (launch_fill(f.data, f.desc.initial_value, c->cells, c->bf16, c->stream) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
            if (launch_fill(f.temp, f.desc.initial_value, c->cells, c->bf16, c->stream) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
        }
        for (auto& f : c->vectors) {
            const float init[3] = {f.desc.initial_value_x, f.desc.initial_value_y, f.desc.initial_value_z};
            for (int k = 0; k < 3; ++k)
                if (init[k] != 0.0f && launch_fill(f.data[k], init[k], c->cells, 0, c->stream) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
        }
    }

    if (build_graph(*c) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    if (cudaGetLastError() != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    *out_context = c.release();
    return STABLE_FLUIDS_RESULT_OK;
}

ScalarField* scalar_field(Context& c, StableFluidsScalarFieldHandle h) {
    if (h == 0 || h > c.scalars.size()) return nullptr;
    return &c.scalars[h - 1u];
}

cudaError_t copy_or_zero(float* dst, const float* src, size_t bytes, cudaStream_t s) {
    return src == nullptr ? cudaMemsetAsync(dst, 0, bytes, s) : cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, s);
}

}  // namespace
}  // namespace sfb

using sfb::Context;

extern "C" {

StableFluidsResult stable_fluids_create_context_cuda(const StableFluidsContextCreateDesc* desc, void** out_context, StableFluidsScalarFieldHandle* out_scalar_field_handles, uint32_t out_scalar_field_handle_capacity, StableFluidsVectorFieldHandle* out_vector_field_handles, uint32_t out_vector_field_handle_capacity) {
    return sfb::create(desc, nullptr, true, out_context, out_scalar_field_handles, out_scalar_field_handle_capacity, out_vector_field_handles, out_vector_field_handle_capacity);
}

StableFluidsResult stable_fluids_b200_create_context(const StableFluidsContextCreateDesc* desc, const StableFluidsB200Options* options, void** out_context, StableFluidsScalarFieldHandle* out_scalar_field_handles, uint32_t out_scalar_field_handle_capacity, StableFluidsVectorFieldHandle* out_vector_field_handles, uint32_t out_vector_field_handle_capacity) {
    return sfb::create(desc, options, false, out_context, out_scalar_field_handles, out_scalar_field_handle_capacity, out_vector_field_handles, out_vector_field_handle_capacity);
}

StableFluidsResult stable_fluids_b200_default_options(StableFluidsB200Options* options) {
    if (options == nullptr) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    sfb::default_options(*options);
    return STABLE_FLUIDS_RESULT_OK;
}

StableFluidsResult stable_fluids_destroy_context_cuda(void* context) {
    sfb::Range range("stable.destroy_context");
    if (context == nullptr) return STABLE_FLUIDS_RESULT_OK;
    auto* c = static_cast<Context*>(context);
    if (c->stream) cudaStreamSynchronize(c->stream);  // :685
    // copies still running on a caller's copy stream into or out of the context
    for (auto& v : c->vectors)
        if (v.stage_ready) cudaEventSynchronize(v.stage_ready);
    if (c->snapshot.used) cudaEventSynchronize(c->snapshot.sent);
    if (c->network != nullptr) sfb::net::release(c->network, c);  // its inference buffers in the attached network
    delete c;
    return STABLE_FLUIDS_RESULT_OK;
}

StableFluidsResult stable_fluids_update_scalar_field_cuda(void* context, StableFluidsScalarFieldHandle field, const float* values) {
    sfb::Range range("stable.update_scalar_field");
    if (context == nullptr) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    auto& c = *static_cast<Context*>(context);
    auto* f = sfb::scalar_field(c, field);
    if (f == nullptr) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    if (c.bf16) {
        // FP32 values through the view copy into BF16 storage
        if (sfb::copy_or_zero(f->view, values, c.field_bytes, c.stream) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
        return sfb::launch_convert(f->data, f->view, c.cells, 1, c.stream) == cudaSuccess ? STABLE_FLUIDS_RESULT_OK : STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    }
    return sfb::copy_or_zero(f->data, values, c.field_bytes, c.stream) == cudaSuccess ? STABLE_FLUIDS_RESULT_OK : STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
}

StableFluidsResult stable_fluids_update_scalar_field_source_cuda(void* context, StableFluidsScalarFieldHandle field, const float* values) {
    sfb::Range range("stable.update_scalar_field_source");
    if (context == nullptr) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    auto& c = *static_cast<Context*>(context);
    auto* f = sfb::scalar_field(c, field);
    if (f == nullptr) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    return sfb::copy_or_zero(f->source, values, c.field_bytes, c.stream) == cudaSuccess ? STABLE_FLUIDS_RESULT_OK : STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
}

StableFluidsResult stable_fluids_update_vector_field_cuda(void* context, StableFluidsVectorFieldHandle field, const float* values_x, const float* values_y, const float* values_z) {
    sfb::Range range("stable.update_vector_field");
    if (context == nullptr) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    auto& c = *static_cast<Context*>(context);
    if (field == 0 || field > c.vectors.size()) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    auto& f = c.vectors[field - 1u];
    const float* src[3] = {values_x, values_y, values_z};
    for (int k = 0; k < 3; ++k)
        if (sfb::copy_or_zero(f.data[k], src[k], c.field_bytes, c.stream) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    return STABLE_FLUIDS_RESULT_OK;
}

StableFluidsResult stable_fluids_step_cuda(void* context) {
    sfb::Range range("stable.step");
    if (context == nullptr) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    auto& c = *static_cast<Context*>(context);
    // staged vector fields: wait for their copies, move them in (device to device)
    for (auto& v : c.vectors) {
        if (!v.staged) continue;
        if (cudaStreamWaitEvent(c.stream, v.stage_ready, 0) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
        for (int k = 0; k < 3; ++k)
            if (cudaMemcpyAsync(v.data[k], v.stage[k], c.field_bytes, cudaMemcpyDeviceToDevice, c.stream) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
        if (cudaEventRecord(v.stage_free, c.stream) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
        v.staged = false;
    }
    return cudaGraphLaunch(c.exec, c.stream) == cudaSuccess ? STABLE_FLUIDS_RESULT_OK : STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
}

StableFluidsResult stable_fluids_b200_stage_vector_field(void* context, StableFluidsVectorFieldHandle field, const float* values_x, const float* values_y, const float* values_z, void* copy_stream) {
    sfb::Range range("stable.stage_vector_field");
    if (context == nullptr || copy_stream == nullptr) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    auto& c = *static_cast<Context*>(context);
    if (field == 0 || field > c.vectors.size()) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    auto& f = c.vectors[field - 1u];
    const auto cs = static_cast<cudaStream_t>(copy_stream);
    if (f.stage[0] == nullptr) {  // first call: the staging arrays and their events
        for (auto*& p : f.stage)
            if (cudaMalloc(reinterpret_cast<void**>(&p), c.field_bytes) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
        if (cudaEventCreateWithFlags(&f.stage_ready, cudaEventDisableTiming) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
        if (cudaEventCreateWithFlags(&f.stage_free, cudaEventDisableTiming) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
        if (cudaEventRecord(f.stage_free, c.stream) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    }
    // a copy staged earlier and not yet taken by a step is replaced; one taken
    // must have left the staging arrays before they are overwritten
    if (cudaStreamWaitEvent(cs, f.stage_free, 0) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    const float* src[3] = {values_x, values_y, values_z};
    for (int k = 0; k < 3; ++k)
        if (sfb::copy_or_zero(f.stage[k], src[k], c.field_bytes, cs) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    if (cudaEventRecord(f.stage_ready, cs) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    f.staged = true;
    return STABLE_FLUIDS_RESULT_OK;
}

StableFluidsResult stable_fluids_get_view_cuda(void* context, const StableFluidsViewRequest* request, StableFluidsView* out_view) {
    sfb::Range range("stable.get_view");
    if (context == nullptr || request == nullptr || out_view == nullptr) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    auto& c = *static_cast<Context*>(context);
    StableFluidsView v{};
    v.layout = STABLE_FLUIDS_VIEW_LAYOUT_F32_3D;
    v.nx = c.config.nx;
    v.ny = c.config.ny;
    v.nz = c.config.nz;
    v.row_stride_bytes = static_cast<uint64_t>(c.config.nx) * sizeof(float);
    v.slice_stride_bytes = static_cast<uint64_t>(c.config.nx) * static_cast<uint64_t>(c.config.ny) * sizeof(float);
    switch (request->kind) {
    case STABLE_FLUIDS_VIEW_SCALAR_FIELD_DATA:
    case STABLE_FLUIDS_VIEW_SCALAR_FIELD_SOURCE: {
        auto* f = sfb::scalar_field(c, request->scalar_field);
        if (f == nullptr) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
        v.data0 = request->kind == STABLE_FLUIDS_VIEW_SCALAR_FIELD_DATA ? f->data : f->source;
        if (c.bf16 && request->kind == STABLE_FLUIDS_VIEW_SCALAR_FIELD_DATA) {
            if (sfb::launch_convert(f->view, f->data, c.cells, 0, c.stream) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
            v.data0 = f->view;
        }
        break;
    }
    case STABLE_FLUIDS_VIEW_VECTOR_FIELD: {
        if (request->vector_field == 0 || request->vector_field > c.vectors.size()) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
        const auto& f = c.vectors[request->vector_field - 1u];
        v.layout = STABLE_FLUIDS_VIEW_LAYOUT_F32_3D_SOA3;
        v.data0 = f.data[0];
        v.data1 = f.data[1];
        v.data2 = f.data[2];
        break;
    }
    case STABLE_FLUIDS_VIEW_FLOW_VELOCITY:
        v.layout = STABLE_FLUIDS_VIEW_LAYOUT_F32_3D_SOA3;
        v.data0 = c.vel[0];
        v.data1 = c.vel[1];
        v.data2 = c.vel[2];
        if (c.bf16) {
            for (int k = 0; k < 3; ++k)
                if (sfb::launch_convert(c.view_vel[k], c.vel[k], c.cells, 0, c.stream) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
            v.data0 = c.view_vel[0];
            v.data1 = c.view_vel[1];
            v.data2 = c.view_vel[2];
        }
        break;
    case STABLE_FLUIDS_VIEW_FLOW_VELOCITY_MAGNITUDE: v.data0 = c.magnitude; break;
    case STABLE_FLUIDS_VIEW_FLOW_PRESSURE: v.data0 = c.pressure; break;
    case STABLE_FLUIDS_VIEW_FLOW_DIVERGENCE: v.data0 = c.divergence; break;
    default: return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;  // :799
    }
    *out_view = v;
    // Order the consumer stream after the work queued so far (:743-759).
    if (request->consumer_stream != nullptr && static_cast<cudaStream_t>(request->consumer_stream) != c.stream) {
        if (cudaEventRecord(c.ready, c.stream) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
        if (cudaStreamWaitEvent(static_cast<cudaStream_t>(request->consumer_stream), c.ready, 0) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    }
    return STABLE_FLUIDS_RESULT_OK;
}

StableFluidsResult stable_fluids_b200_read_view_async(void* context, const StableFluidsViewRequest* request, float* host_out0, float* host_out1, float* host_out2, void* copy_stream) {
    sfb::Range range("stable.read_view_async");
    if (context == nullptr || request == nullptr || copy_stream == nullptr || host_out0 == nullptr) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    auto& c = *static_cast<Context*>(context);
    StableFluidsViewRequest r = *request;
    r.consumer_stream = nullptr;
    StableFluidsView v{};
    if (stable_fluids_get_view_cuda(context, &r, &v) != STABLE_FLUIDS_RESULT_OK) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    const int arrays = v.layout == STABLE_FLUIDS_VIEW_LAYOUT_F32_3D_SOA3 ? 3 : 1;
    float* const out[3] = {host_out0, host_out1, host_out2};
    const void* const in[3] = {v.data0, v.data1, v.data2};
    for (int k = 0; k < arrays; ++k)
        if (out[k] == nullptr) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    auto& sn = c.snapshot;
    const auto cs = static_cast<cudaStream_t>(copy_stream);
    if (sn.taken == nullptr) {
        if (cudaEventCreateWithFlags(&sn.taken, cudaEventDisableTiming) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
        if (cudaEventCreateWithFlags(&sn.sent, cudaEventDisableTiming) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    }
    for (int k = 0; k < arrays; ++k)
        if (sn.snap[k] == nullptr && cudaMalloc(reinterpret_cast<void**>(&sn.snap[k]), c.field_bytes) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    // the previous read-back must have left the snapshot before it is overwritten
    if (sn.used && cudaStreamWaitEvent(c.stream, sn.sent, 0) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    for (int k = 0; k < arrays; ++k)
        if (cudaMemcpyAsync(sn.snap[k], in[k], c.field_bytes, cudaMemcpyDeviceToDevice, c.stream) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    if (cudaEventRecord(sn.taken, c.stream) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    if (cudaStreamWaitEvent(cs, sn.taken, 0) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    for (int k = 0; k < arrays; ++k)
        if (cudaMemcpyAsync(out[k], sn.snap[k], c.field_bytes, cudaMemcpyDeviceToHost, cs) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    if (cudaEventRecord(sn.sent, cs) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    sn.used = true;
    return STABLE_FLUIDS_RESULT_OK;
}

StableFluidsResult stable_fluids_b200_get_step_stats(void* context, StableFluidsB200StepStats* out_stats) {
    if (context == nullptr || out_stats == nullptr) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    auto& c = *static_cast<Context*>(context);
    if (cudaMemcpyAsync(c.host_stats, c.stats, sizeof(sfb::DeviceStats), cudaMemcpyDeviceToHost, c.stream) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    if (cudaStreamSynchronize(c.stream) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    const auto& d = *c.host_stats;
    StableFluidsB200StepStats o{};
    o.rel_residual = c.residual_enabled ? d.rel_residual : -1.0;
    o.rhs_norm = c.residual_enabled ? d.rhs_norm : 0.0;
    o.pressure_iterations = c.residual_enabled ? d.iterations : c.config.pressure_iterations;
    o.hit_cap = d.hit_cap;
    // a learned-start context without a network runs the previous-pressure start
    const bool learned = c.options.warm_start == STABLE_FLUIDS_B200_WARM_START_LEARNED;
    o.used_fallback = learned ? (c.network == nullptr ? 1 : d.used_fallback) : 0;
    *out_stats = o;
    return STABLE_FLUIDS_RESULT_OK;
}

}  // extern "C"

extern "C" {

StableFluidsResult stable_fluids_b200_enqueue_stage(void* context, uint32_t stage, int32_t* out_kernel_launches) {
    if (context == nullptr) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    auto& c = *static_cast<Context*>(context);
    sfb::Stages st{c};
    switch (stage) {
    case STABLE_FLUIDS_B200_STAGE_FORCES: st.forces(); break;
    case STABLE_FLUIDS_B200_STAGE_VELOCITY_ADVECTION: st.advect_velocity(); break;
    case STABLE_FLUIDS_B200_STAGE_VELOCITY_DIFFUSION: st.diffuse_velocity(); break;
    case STABLE_FLUIDS_B200_STAGE_DIVERGENCE: st.divergence(); break;
    case STABLE_FLUIDS_B200_STAGE_PRESSURE: st.pressure(); break;
    case STABLE_FLUIDS_B200_STAGE_PROJECTION: st.project(); break;
    case STABLE_FLUIDS_B200_STAGE_SCALARS: st.scalars(); break;
    case STABLE_FLUIDS_B200_STAGE_DIAGNOSTICS: st.diagnostics(); break;
    case STABLE_FLUIDS_B200_STAGE_STEP:
        if (cudaGraphLaunch(c.exec, c.stream) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
        st.launches = c.step_kernels;
        break;
    default: return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    }
    if (st.e != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    if (out_kernel_launches) *out_kernel_launches = st.launches;
    return STABLE_FLUIDS_RESULT_OK;
}

// The viewer's plume geometry from the context's grid (scene_plume.cpp:229-246),
// in the same float expressions.
static sfb::PlumeGeometry plume_geometry(const Context& c) {
    sfb::PlumeGeometry g{};
    const float h = c.config.cell_size;
    const float extent_x = static_cast<float>(c.dims.nx) * h;
    const float extent_y = static_cast<float>(c.dims.ny) * h;
    const float extent_z = static_cast<float>(c.dims.nz) * h;
    g.h = h;
    g.source_x = extent_x * 0.50f;
    g.source_y = extent_y * 0.13f;
    g.source_z = extent_z * 0.50f;
    g.source_r = h * 6.0f;
    g.swirl_y = g.source_y + g.source_r * 0.90f;
    g.drift_y = g.source_y + g.source_r * 1.35f;
    g.swirl_r = g.source_r * 1.65f;
    g.drift_r = g.source_r * 2.10f;
    return g;
}

StableFluidsResult stable_fluids_b200_plume_scene_setup(void* context, StableFluidsScalarFieldHandle density, StableFluidsVectorFieldHandle force) {
    if (context == nullptr) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    auto& c = *static_cast<Context*>(context);
    auto* f = sfb::scalar_field(c, density);
    if (f == nullptr || force == 0 || force > c.vectors.size()) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    auto& v = c.vectors[force - 1u];
    return sfb::launch_plume_setup(f->source, v.data[0], v.data[1], v.data[2], plume_geometry(c), c.dims, c.stream) == cudaSuccess ? STABLE_FLUIDS_RESULT_OK : STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
}

StableFluidsResult stable_fluids_b200_plume_scene_forces(void* context, StableFluidsVectorFieldHandle force, int32_t animation_step) {
    if (context == nullptr) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    auto& c = *static_cast<Context*>(context);
    if (force == 0 || force > c.vectors.size()) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    auto& v = c.vectors[force - 1u];
    // the animated scalars as the viewer computes them (scene_plume.cpp:323-326)
    const float phase = static_cast<float>(animation_step) * 0.045f;
    const float drift_x = 1.15f * std::sin(phase);
    const float drift_z = 0.85f * std::cos(phase * 0.71f);
    const float swirl = 1.65f * std::cos(phase * 0.53f);
    return sfb::launch_plume_forces(v.data[0], v.data[2], plume_geometry(c), c.dims, drift_x, drift_z, swirl, c.stream) == cudaSuccess ? STABLE_FLUIDS_RESULT_OK : STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
}

StableFluidsResult stable_fluids_b200_render_volume(void* context, const StableFluidsViewRequest* field, const StableFluidsB200VolumeRender* params, float* out_rgba) {
    sfb::Range range("stable.render_volume");
    if (context == nullptr || field == nullptr || params == nullptr || out_rgba == nullptr) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    if (params->width <= 0 || params->height <= 0 || params->width > 16384 || params->height > 16384) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    auto& c = *static_cast<Context*>(context);
    StableFluidsView v{};
    const StableFluidsResult r = stable_fluids_get_view_cuda(context, field, &v);
    if (r != STABLE_FLUIDS_RESULT_OK) return r;
    if (v.layout != STABLE_FLUIDS_VIEW_LAYOUT_F32_3D || v.data0 == nullptr) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;  // one array only
    sfb::RenderParams p{};
    for (int k = 0; k < 3; ++k) {
        p.eye[k] = params->eye[k];
        p.right[k] = params->right[k];
        p.up[k] = params->up[k];
        p.forward[k] = params->forward[k];
        p.volume_min[k] = params->volume_min[k];
        p.volume_max[k] = params->volume_max[k];
        p.color_a[k] = params->color_a[k];
        p.color_b[k] = params->color_b[k];
    }
    p.aspect = params->aspect;
    p.tan_half_fov = params->tan_half_fov;
    p.value_scale = params->value_scale;
    p.density = params->density;
    p.value_min = params->value_min;
    p.value_max = params->value_max;
    p.ortho_height = params->ortho_height;
    p.steps = params->steps;
    p.projection = params->projection;
    p.width = params->width;
    p.height = params->height;
    return sfb::launch_render_volume(static_cast<const float*>(v.data0), c.dims, p, out_rgba, c.stream) == cudaSuccess ? STABLE_FLUIDS_RESULT_OK : STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
}

StableFluidsResult stable_fluids_b200_attach_network(void* context, void* network) {
    if (context == nullptr) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    auto& c = *static_cast<Context*>(context);
    if (c.options.warm_start != STABLE_FLUIDS_B200_WARM_START_LEARNED) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    auto* n = static_cast<sfb::net::Net*>(network);
    if (cudaStreamSynchronize(c.stream) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    // the network's buffers for this grid are allocated before the capture
    if (n != nullptr && sfb::net::prepare(n, c.coarse_b != nullptr ? c.coarse_dims() : c.dims, &c) != cudaSuccess) {
        cudaGetLastError();
        return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    }
    sfb::net::Net* const previous = c.network;
    c.network = n;
    if (sfb::build_graph(c) != cudaSuccess) {
        c.network = previous;
        sfb::build_graph(c);  // put the previous step graph back
        return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    }
    // the new step graph no longer uses the previous network's buffers for this context
    if (previous != nullptr && previous != n) sfb::net::release(previous, &c);
    return STABLE_FLUIDS_RESULT_OK;
}

}  // extern "C"

namespace sfb {
namespace {

// A batch of contexts stepped together (stable-fluids-b200.h).
//  GRAPHS: the contexts' step graphs as child graphs of one graph, launched
//    once per batch step; the children share no data, so the GPU runs the
//    simulations' kernels concurrently.
//  WORK_TABLE: one graph of persistent launches, one per stage of the step,
//    each covering every simulation through the work table (sf_batch.h).
struct Batch {
    std::vector<Context*> contexts;
    cudaStream_t stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t done = nullptr;
    int kernels = 0;
    uint32_t mode = STABLE_FLUIDS_B200_BATCH_GRAPHS;
    // work table: host entries (grouped: the simulations of a group are
    // contiguous), their device copy, the per-group per-shape prefix offsets,
    // and one table per group
    std::vector<BatchSim> sims;
    std::vector<int> order;                      // sims[i] belongs to context order[i]
    std::vector<std::pair<int, int>> groups;     // [begin, end) ranges of sims
    BatchSim* d_sims = nullptr;
    uint32_t* d_first = nullptr;
    std::vector<BatchTable> tables;              // one per group
    int chains = 1;                              // groups captured round-robin on this many concurrent streams
    std::vector<cudaStream_t> chain_streams;     // chains - 1 extra capture streams
    std::vector<cudaEvent_t> chain_events;       // fork + one join event per extra stream
    bool rb_split = false;                       // red-black solves in the colour-split layout

    ~Batch() {
        for (auto ev : chain_events) cudaEventDestroy(ev);
        for (auto st : chain_streams) cudaStreamDestroy(st);
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (done) cudaEventDestroy(done);
        if (stream) cudaStreamDestroy(stream);
        if (d_sims) cudaFree(d_sims);
        if (d_first) cudaFree(d_first);
    }
};

float alpha_velocity(const Context& c) {
    const float h = c.config.cell_size;
    return c.config.dt * c.config.viscosity / (h * h);  // same expression as Stages::alpha_v
}
float alpha_scalar(const Context& c, const ScalarField& f) {
    const float h = c.config.cell_size;
    return c.config.dt * f.desc.diffusion / (h * h);  // same expression as Stages::alpha_s
}
int force_fields(const Context& c) {
    int n = 0;
    for (const auto& v : c.vectors) n += v.desc.usage == STABLE_FLUIDS_VECTOR_FIELD_FORCE ? 1 : 0;
    return n;
}

// Whether the contexts share the stage structure the work-table kernels
// implement (one step = the same sequence of stages and sweep counts).
bool work_table_compatible(const std::vector<Context*>& cs) {
    const Context& r = *cs.front();
    for (const Context* c : cs) {
        const auto& o = c->options;
        if (c->bf16 || c->blocked || c->network != nullptr) return false;
        if (o.scheme != r.options.scheme || o.warm_start != r.options.warm_start || o.warm_start == STABLE_FLUIDS_B200_WARM_START_LEARNED) return false;
        if (o.residual_tolerance > 0.0f || c->residual_enabled != r.residual_enabled) return false;
        if (c->config.diffuse_iterations != r.config.diffuse_iterations || c->config.pressure_iterations != r.config.pressure_iterations) return false;
        if (!(alpha_velocity(*c) > 0.0f) || c->scalars.size() != 1 || !(alpha_scalar(*c, c->scalars[0]) > 0.0f)) return false;
        if ((c->scalars[0].desc.dissipation > 0.0f) != (r.scalars[0].desc.dissipation > 0.0f)) return false;
        if (force_fields(*c) > kBatchForces) return false;
        if (c->dims.nx % 4 != 0 || c->cells >= (1ull << 31)) return false;
    }
    return true;
}

BatchSim make_batch_sim(const Context& c, int z_chunk) {
    BatchSim m{};
    const ScalarField& f = c.scalars[0];
    m.d = c.dims;
    m.h = c.config.cell_size;
    m.dt = c.config.dt;
    m.alpha_v = alpha_velocity(c);
    m.alpha_s = alpha_scalar(c, f);
    m.scale_s = f.desc.dissipation > 0.0f ? 1.0f / (1.0f + c.config.dt * f.desc.dissipation) : 1.0f;
    m.z_chunk = z_chunk;
    m.flow = c.flow;
    m.sbc = f.bc;
    for (int k = 0; k < 5; ++k) m.ghost[k] = make_ghost_rule(k, c.flow, k == KIND_SCALAR ? f.bc : ScalarBC{});
    for (int k = 0; k < 3; ++k) {
        m.vel[k] = c.vel[k];
        m.temp[k] = c.temp[k];
    }
    m.packed = static_cast<float*>(c.packed);
    m.pressure = c.pressure;
    m.divergence = c.divergence;
    m.magnitude = c.magnitude;
    m.scratch = c.scratch;
    m.scratch2 = c.scratch2;
    m.sdata = f.data;
    m.stemp = f.temp;
    m.source = f.source;
    for (const auto& v : c.vectors) {
        if (v.desc.usage != STABLE_FLUIDS_VECTOR_FIELD_FORCE) continue;
        for (int k = 0; k < 3; ++k) m.force[m.force_count][k] = v.data[k];
        ++m.force_count;
    }
    m.stats = c.stats;
    return m;
}

// Uploads the entries and, per group, the prefix offsets per launch shape.
cudaError_t upload_table(Batch& b) {
    const int n = static_cast<int>(b.sims.size());
    const int ng = static_cast<int>(b.groups.size());
    std::vector<uint32_t> first(kBatchShapes * static_cast<size_t>(n + ng));
    b.tables.assign(ng, BatchTable{});
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    size_t at = 0;
    std::vector<size_t> offset(kBatchShapes * static_cast<size_t>(ng));
    for (int g = 0; g < ng; ++g) {
        const auto [lo, hi] = b.groups[g];
        for (int shape = 0; shape < kBatchShapes; ++shape) {
            offset[kBatchShapes * g + shape] = at;
            uint32_t acc = 0;
            for (int i = lo; i < hi; ++i) {
                first[at++] = acc;
                acc += batch_blocks(b.sims[i].d, shape, b.sims[i].z_chunk);
            }
            first[at++] = acc;
            b.tables[g].total[shape] = acc;
        }
    }
    cudaError_t e = cudaSuccess;
    if (b.d_sims == nullptr && (e = cudaMalloc(&b.d_sims, sizeof(BatchSim) * n)) != cudaSuccess) return e;
    if (b.d_first == nullptr && (e = cudaMalloc(&b.d_first, sizeof(uint32_t) * first.size())) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(b.d_sims, b.sims.data(), sizeof(BatchSim) * n, cudaMemcpyHostToDevice, b.stream)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(b.d_first, first.data(), sizeof(uint32_t) * first.size(), cudaMemcpyHostToDevice, b.stream)) != cudaSuccess) return e;
    if ((e = cudaStreamSynchronize(b.stream)) != cudaSuccess) return e;
    for (int g = 0; g < ng; ++g) {
        auto& t = b.tables[g];
        t.sims = b.d_sims + b.groups[g].first;
        for (int shape = 0; shape < kBatchShapes; ++shape) t.first[shape] = b.d_first + offset[kBatchShapes * g + shape];
        t.nsims = b.groups[g].second - b.groups[g].first;
        t.sms = sms;
    }
    return cudaSuccess;
}

// Groups of simulations whose sweep working set (iterate, right-hand side
// and scratch: 12 bytes per cell) fits in half the L2 cache divided among the
// concurrent chains: each chain runs its groups one after another, so a
// group's hundreds of sweeps reread its fields from L2 instead of HBM. Largest simulations first, first fit. Fills
// b.sims / b.order / b.groups; `make` builds one entry from a context index.
template <typename Make>
void group_by_l2(Batch& b, Make make) {
    int dev = 0, l2 = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev) != cudaSuccess || l2 <= 0) l2 = 50 << 20;
    const size_t budget = static_cast<size_t>(l2) / 2 / 12 / static_cast<size_t>(b.chains);  // cells per group (chains run concurrently)
    std::vector<int> idx(b.contexts.size());
    for (size_t i = 0; i < idx.size(); ++i) idx[i] = static_cast<int>(i);
    std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return b.contexts[x]->cells > b.contexts[y]->cells; });
    std::vector<std::vector<int>> bins;
    std::vector<size_t> fill;
    for (int i : idx) {
        const size_t c = b.contexts[i]->cells;
        size_t k = 0;
        while (k < bins.size() && fill[k] + c > budget) ++k;
        if (k == bins.size()) {
            bins.emplace_back();
            fill.push_back(0);
        }
        bins[k].push_back(i);
        fill[k] += c;
    }
    b.sims.clear();
    b.order.clear();
    b.groups.clear();
    for (const auto& bin : bins) {
        const int lo = static_cast<int>(b.sims.size());
        for (int i : bin) {
            b.sims.push_back(make(i));
            b.order.push_back(i);
        }
        b.groups.emplace_back(lo, static_cast<int>(b.sims.size()));
    }
}

// ---- tile autotuner ------------------------------------------------------
// The z chunk (planes per thread block) of the vectorised sweeps, per grid
// size: each candidate is timed on the whole batch with CUDA events (a Jacobi
// pressure sweep from the pressure into the scratch buffer, so no simulation
// state changes), one size class at a time with the others fixed. Results
// are kept in a flat JSON object {"<gpu>|<nx>x<ny>x<nz>": z_chunk, ...}.
constexpr int kDefaultZChunk = 16;
constexpr int kDefaultChains = 4;  // concurrent group chains of a work-table batch (measured best on B200: 3-4)

std::string tile_key(const std::string& gpu, const Dims& d) { return gpu + "|" + std::to_string(d.nx) + "x" + std::to_string(d.ny) + "x" + std::to_string(d.nz); }

std::vector<std::pair<std::string, int>> read_tile_cache(const char* path) {
    std::vector<std::pair<std::string, int>> out;
    if (path == nullptr) return out;
    std::FILE* f = std::fopen(path, "rb");
    if (f == nullptr) return out;
    std::string text;
    char buf[4096];
    size_t got;
    while ((got = std::fread(buf, 1, sizeof(buf), f)) > 0) text.append(buf, got);
    std::fclose(f);
    // "key": value pairs of a flat object; anything else is ignored
    size_t i = 0;
    while ((i = text.find('"', i)) != std::string::npos) {
        const size_t j = text.find('"', i + 1);
        if (j == std::string::npos) break;
        const std::string key = text.substr(i + 1, j - i - 1);
        size_t k = text.find_first_not_of(" \t\r\n", j + 1);
        if (k == std::string::npos || text[k] != ':') {
            i = j + 1;
            continue;
        }
        k = text.find_first_not_of(" \t\r\n", k + 1);
        if (k == std::string::npos) break;
        char* end = nullptr;
        const long v = std::strtol(text.c_str() + k, &end, 10);
        if (end != text.c_str() + k && v > 0 && v < (1 << 20)) out.emplace_back(key, static_cast<int>(v));
        i = static_cast<size_t>(end - text.c_str());
        if (i <= j) i = j + 1;
    }
    return out;
}

void write_tile_cache(const char* path, const std::vector<std::pair<std::string, int>>& entries) {
    if (path == nullptr) return;
    std::FILE* f = std::fopen(path, "wb");
    if (f == nullptr) return;
    std::fputs("{\n", f);
    for (size_t i = 0; i < entries.size(); ++i) std::fprintf(f, "  \"%s\": %d%s\n", entries[i].first.c_str(), entries[i].second, i + 1 < entries.size() ? "," : "");
    std::fputs("}\n", f);
    std::fclose(f);
}

// Average duration of `repeats` batched Jacobi pressure sweeps (scratch <-
// update(p)) per group, summed over the groups, as the step runs them.
float time_batch_sweep(Batch& b, int repeats) {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return -1.0f;
    float ms = -1.0f;
    if (cudaEventRecord(e0, b.stream) == cudaSuccess) {
        bool ok = true;
        for (const auto& t : b.tables)
            for (int r = 0; r < repeats; ++r) ok = ok && launch_batch_sweep(t, KIND_PRESSURE, SCHEME_JACOBI, 0, BF_SCRATCH, BF_X, b.stream) == cudaSuccess;
        if (ok && cudaEventRecord(e1, b.stream) == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return ms < 0.0f ? -1.0f : ms / static_cast<float>(repeats);
}

cudaError_t tune_tiles(Batch& b, const char* cache_path) {
    int dev = 0;
    cudaDeviceProp prop{};
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaGetDeviceProperties(&prop, dev);
    if (e != cudaSuccess) return e;
    const std::string gpu = prop.name;
    auto cache = read_tile_cache(cache_path);
    const auto lookup = [&](const std::string& k) -> int {
        for (const auto& [key, v] : cache)
            if (key == k) return v;
        return 0;
    };
    // size classes in first-seen order
    std::vector<Dims> classes;
    for (const auto& m : b.sims) {
        bool seen = false;
        for (const auto& d : classes) seen = seen || (d.nx == m.d.nx && d.ny == m.d.ny && d.nz == m.d.nz);
        if (!seen) classes.push_back(m.d);
    }
    const auto set_class = [&](const Dims& d, int zc) {
        for (auto& m : b.sims)
            if (m.d.nx == d.nx && m.d.ny == d.ny && m.d.nz == d.nz) m.z_chunk = std::min(zc, d.nz);
    };
    std::vector<Dims> todo;
    for (const auto& d : classes) {
        const int cached = lookup(tile_key(gpu, d));
        if (cached > 0) set_class(d, cached);
        else todo.push_back(d);
    }
    if (!todo.empty()) {
        if ((e = upload_table(b)) != cudaSuccess) return e;
        time_batch_sweep(b, 2);  // warm-up
        for (const Dims& d : todo) {
            int best = std::min(kDefaultZChunk, d.nz);
            float best_ms = -1.0f;
            for (int zc : {2, 4, 8, 16, 32, 64, 128, 256}) {
                if (zc > d.nz) break;
                set_class(d, zc);
                if ((e = upload_table(b)) != cudaSuccess) return e;
                const float ms = time_batch_sweep(b, 5);
                if (ms > 0.0f && (best_ms < 0.0f || ms < best_ms)) {
                    best_ms = ms;
                    best = zc;
                }
            }
            set_class(d, best);
            cache.emplace_back(tile_key(gpu, d), best);
        }
        write_tile_cache(cache_path, cache);
    }
    return upload_table(b);
}

// ---- the batched step -------------------------------------------------------
// The stages of Stages::whole_step in the same order with the same sweep
// counts and buffer sequence, each as one work-table launch.
struct BatchStages {
    Batch& b;
    const BatchTable& t;  // the group's work table
    const Context& r;     // every context has r's stage structure
    cudaStream_t s;       // the capture stream of the group's chain
    cudaError_t e = cudaSuccess;
    int launches = 0;

    void ok(cudaError_t x) {
        if (x == cudaSuccess) ++launches;
        else if (e == cudaSuccess) e = x;
    }

    // One solve: the buffer sequence of run_simple (no temporal blocking);
    // `dissipate`: multiply the scalar by its dissipation factor afterwards.
    void solve(int kind, int init, int iterations, bool dissipate = false) {
        if (r.options.scheme == STABLE_FLUIDS_B200_SCHEME_RBGS && b.rb_split && iterations > 0) {
            // colour-split layout (run_rb_split); the merge applies the dissipation
            ok(launch_batch_rb_split(t, kind, BF_B, init == INIT_FROM_B ? 1 : 0, s));
            if (init == INIT_ZERO) ok(launch_batch_copy(t, kind, BF_SCRATCH, -1, s));
            else if (init == INIT_FROM_X) ok(launch_batch_rb_split(t, kind, BF_X, 0, s));
            for (int it = 0; it < iterations; ++it)
                for (int colour = 0; colour < 2; ++colour) ok(launch_batch_rb_half(t, kind, colour, s));
            ok(launch_batch_rb_merge(t, kind, dissipate ? 1 : 0, s));
            return;
        }
        solve_plain(kind, init, iterations);
        if (dissipate) ok(launch_batch_scale_scalar(t, s));
    }

    void solve_plain(int kind, int init, int iterations) {
        if (r.options.scheme == STABLE_FLUIDS_B200_SCHEME_RBGS) {
            if (init == INIT_FROM_B) ok(launch_batch_copy(t, kind, BF_X, BF_B, s));
            else if (init == INIT_ZERO) ok(launch_batch_copy(t, kind, BF_X, -1, s));
            for (int it = 0; it < iterations; ++it)
                for (int parity = 0; parity < 2; ++parity) ok(launch_batch_sweep(t, kind, SCHEME_RBGS, parity, BF_X, BF_X, s));
            return;
        }
        int src = BF_X;
        if (init == INIT_FROM_B) src = BF_B;
        else if (init == INIT_ZERO) {
            const int zero = (iterations & 1) ? BF_SCRATCH : BF_X;
            ok(launch_batch_copy(t, kind, zero, -1, s));
            src = zero;
        }
        if (iterations == 0) {
            if (src != BF_X) ok(launch_batch_copy(t, kind, BF_X, src, s));
            return;
        }
        for (int u = 0; u < iterations; ++u) {
            const int left = iterations - u;
            int dst = (left & 1) ? BF_X : BF_SCRATCH;
            if (dst == src) dst = dst == BF_X ? BF_SCRATCH : BF_X;
            ok(launch_batch_sweep(t, kind, SCHEME_JACOBI, 0, dst, src, s));
            src = dst;
        }
        if (src != BF_X) ok(launch_batch_copy(t, kind, BF_X, src, s));
    }

    cudaError_t whole_step() {
        const int diffuse = r.config.diffuse_iterations, pressure = r.config.pressure_iterations;
        ok(launch_batch_force_pack(t, s));
        ok(launch_batch_advect_velocity(t, s));
        for (int comp = 0; comp < 3; ++comp) solve(KIND_VEL_X + comp, INIT_FROM_B, diffuse);
        ok(launch_batch_divergence(t, s));
        solve(KIND_PRESSURE, r.options.warm_start == STABLE_FLUIDS_B200_WARM_START_ZERO ? INIT_ZERO : INIT_FROM_X, pressure);
        ok(launch_batch_project(t, 1, s));
        if (r.residual_enabled) {
            ok(launch_batch_stats(t, 0, 0, s));
            ok(launch_batch_residual_sums(t, s));
            ok(launch_batch_stats(t, 1, pressure, s));
        }
        ok(launch_batch_scalar_source_advect(t, s));
        solve(KIND_SCALAR, INIT_FROM_B, diffuse, r.scalars[0].desc.dissipation > 0.0f);
        ok(launch_batch_post_diagnostics(t, s));
        return e;
    }
};

cudaError_t build_work_table(Batch& b, bool autotune, const char* cache_path, int chains) {
    b.chains = std::max(1, std::min(chains, 8));
    cudaError_t e = cudaSuccess;
    for (int c = 1; c < b.chains; ++c) {
        cudaStream_t st = nullptr;
        if ((e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) != cudaSuccess) return e;
        b.chain_streams.push_back(st);
    }
    for (int c = 0; c < b.chains; ++c) {  // [0] forks the chains, [c] joins chain c
        cudaEvent_t ev = nullptr;
        if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) return e;
        b.chain_events.push_back(ev);
    }
    // red-black solves in the colour-split layout when every simulation allows it
    b.rb_split = true;
    for (const Context* c : b.contexts) {
        const ScalarBC& sb = c->scalars[0].bc;
        const int n[3] = {c->dims.nx, c->dims.ny, c->dims.nz};
        bool ok = c->scratch2 != nullptr && c->dims.nx % 8 == 0;
        for (int k = 0; k < 3; ++k) ok = ok && !((c->flow.periodic[k] || sb.periodic[k]) && (n[k] & 1));
        b.rb_split = b.rb_split && ok;
    }
    group_by_l2(b, [&](int i) { return make_batch_sim(*b.contexts[i], std::min(kDefaultZChunk, b.contexts[i]->dims.nz)); });
    e = autotune ? tune_tiles(b, cache_path) : upload_table(b);
    if (e != cudaSuccess) return e;
    if ((e = cudaStreamBeginCapture(b.stream, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) return e;
    cudaError_t rec = cudaSuccess;
    const auto step = [&](cudaError_t x) {
        if (rec == cudaSuccess) rec = x;
    };
    if (b.chains > 1) {
        step(cudaEventRecord(b.chain_events[0], b.stream));
        for (auto st : b.chain_streams) step(cudaStreamWaitEvent(st, b.chain_events[0], 0));
    }
    b.kernels = 0;
    for (size_t g = 0; g < b.tables.size(); ++g) {  // chain c runs groups c, c + chains, ...: each group's step reuses L2
        const size_t c = g % static_cast<size_t>(b.chains);
        BatchStages st{b, b.tables[g], *b.contexts.front(), c == 0 ? b.stream : b.chain_streams[c - 1]};
        if (rec == cudaSuccess) rec = st.whole_step();
        b.kernels += st.launches;
    }
    for (int c = 1; c < b.chains; ++c) {
        step(cudaEventRecord(b.chain_events[c], b.chain_streams[c - 1]));
        step(cudaStreamWaitEvent(b.stream, b.chain_events[c], 0));
    }
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(b.stream, &g);
    if (rec != cudaSuccess || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return rec != cudaSuccess ? rec : e;
    }
    b.graph = g;
    return cudaSuccess;
}

cudaError_t build_child_graphs(Batch& b) {
    // The children run concurrently; contexts attached to one warm-start
    // network each predict with activation buffers of their own and share
    // its weights, which no step writes.
    cudaError_t e = cudaGraphCreate(&b.graph, 0);
    if (e != cudaSuccess) return e;
    for (Context* c : b.contexts) {
        if (c->graph == nullptr) return cudaErrorInvalidValue;
        cudaGraphNode_t node = nullptr;
        if ((e = cudaGraphAddChildGraphNode(&node, b.graph, nullptr, 0, c->graph)) != cudaSuccess) return e;
        b.kernels += c->step_kernels;
    }
    return cudaSuccess;
}

}  // namespace
}  // namespace sfb

extern "C" {

StableFluidsResult stable_fluids_b200_batch_create(void* const* contexts, uint32_t count, void** out_batch) {
    StableFluidsB200BatchOptions o{};  // GRAPHS, no autotuning
    return stable_fluids_b200_batch_create_ex(contexts, count, &o, out_batch);
}

StableFluidsResult stable_fluids_b200_batch_create_ex(void* const* contexts, uint32_t count, const StableFluidsB200BatchOptions* options, void** out_batch) {
    sfb::Range range("stable.batch_create");
    if (out_batch == nullptr) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    *out_batch = nullptr;
    if (contexts == nullptr || count == 0 || options == nullptr || options->mode > STABLE_FLUIDS_B200_BATCH_WORK_TABLE) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    std::unique_ptr<sfb::Batch> b{new (std::nothrow) sfb::Batch{}};
    if (!b) return STABLE_FLUIDS_RESULT_OUT_OF_MEMORY;
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    if (cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    for (uint32_t i = 0; i < count; ++i) {
        auto* c = static_cast<Context*>(contexts[i]);
        if (c == nullptr || c->graph == nullptr) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
        for (auto* other : b->contexts)
            if (other == c) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;  // a context steps once per batch step
        // all work queued on the context so far (updates) precedes the batch
        if (cudaStreamSynchronize(c->stream) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
        b->contexts.push_back(c);
    }
    cudaError_t e;
    if (options->mode == STABLE_FLUIDS_B200_BATCH_WORK_TABLE) {
        if (!sfb::work_table_compatible(b->contexts)) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
        b->mode = STABLE_FLUIDS_B200_BATCH_WORK_TABLE;
        e = sfb::build_work_table(*b, options->autotune != 0, options->tile_cache, options->chains == 0 ? sfb::kDefaultChains : static_cast<int>(options->chains));
    } else {
        b->mode = STABLE_FLUIDS_B200_BATCH_GRAPHS;
        e = sfb::build_child_graphs(*b);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        return e == cudaErrorMemoryAllocation ? STABLE_FLUIDS_RESULT_OUT_OF_MEMORY : STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    }
    if (cudaGraphInstantiate(&b->exec, b->graph, 0) != cudaSuccess) {
        b->exec = nullptr;
        cudaGetLastError();
        return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    }
    *out_batch = b.release();
    return STABLE_FLUIDS_RESULT_OK;
}

StableFluidsResult stable_fluids_b200_batch_layout(void* batch, uint32_t* out_mode, uint32_t* out_groups, int32_t* out_z_chunks, uint32_t capacity) {
    if (batch == nullptr) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    const auto& b = *static_cast<const sfb::Batch*>(batch);
    if (out_mode) *out_mode = b.mode;
    if (out_groups) *out_groups = static_cast<uint32_t>(b.groups.size());
    if (out_z_chunks) {
        for (uint32_t i = 0; i < capacity && i < b.contexts.size(); ++i) out_z_chunks[i] = 0;
        for (size_t k = 0; k < b.sims.size(); ++k)
            if (static_cast<uint32_t>(b.order[k]) < capacity) out_z_chunks[b.order[k]] = b.sims[k].z_chunk;
    }
    return STABLE_FLUIDS_RESULT_OK;
}

StableFluidsResult stable_fluids_b200_batch_step(void* batch) {
    sfb::Range range("stable.batch_step");
    if (batch == nullptr) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    auto& b = *static_cast<sfb::Batch*>(batch);
    // order the batch after each context's queued work and each context after the batch
    for (auto* c : b.contexts) {
        if (cudaEventRecord(c->ready, c->stream) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
        if (cudaStreamWaitEvent(b.stream, c->ready, 0) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    }
    if (cudaGraphLaunch(b.exec, b.stream) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    if (cudaEventRecord(b.done, b.stream) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    for (auto* c : b.contexts)
        if (cudaStreamWaitEvent(c->stream, b.done, 0) != cudaSuccess) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    return STABLE_FLUIDS_RESULT_OK;
}

StableFluidsResult stable_fluids_b200_batch_info(void* batch, uint32_t* out_count, int32_t* out_kernels_per_step, void** out_stream) {
    if (batch == nullptr) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    const auto& b = *static_cast<const sfb::Batch*>(batch);
    if (out_count) *out_count = static_cast<uint32_t>(b.contexts.size());
    if (out_kernels_per_step) *out_kernels_per_step = b.kernels;
    if (out_stream) *out_stream = b.stream;
    return STABLE_FLUIDS_RESULT_OK;
}

StableFluidsResult stable_fluids_b200_batch_destroy(void* batch) {
    if (batch == nullptr) return STABLE_FLUIDS_RESULT_OK;
    auto* b = static_cast<sfb::Batch*>(batch);
    if (b->stream) cudaStreamSynchronize(b->stream);
    delete b;
    return STABLE_FLUIDS_RESULT_OK;
}

StableFluidsResult stable_fluids_b200_get_step_info(void* context, StableFluidsB200StepInfo* out_info) {
    if (context == nullptr || out_info == nullptr) return STABLE_FLUIDS_RESULT_BACKEND_FAILURE;
    const auto& c = *static_cast<const Context*>(context);
    StableFluidsB200StepInfo o{};
    o.kernels_per_step = c.step_kernels;
    o.device_bytes = c.slab_bytes;
    o.scheme = c.options.scheme;
    o.iterations_per_pass = c.options.iterations_per_pass;
    o.blocked = c.blocked ? 1 : 0;
    o.kernels_per_check = c.check_kernels;
    *out_info = o;
    return STABLE_FLUIDS_RESULT_OK;
}

}  // extern "C"
