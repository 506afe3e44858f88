// sf_oracle.cpp -- CPU restatement of the reference stable-fluids step.
//
// TEST INFRASTRUCTURE ONLY. This is the checker, never the product: only
// tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
// The product (libstable-fluids.so) never links or calls anything here.
//
// It restates, in plain C++ on the host, the arithmetic and stage order of
// Xayah-Graphics/stable-fluids backend-cuda.cu:
//   - ghost rules            backend-cuda.cu:62-189
//   - trilinear sampling     backend-cuda.cu:191-293
//   - RK2 back-trace         backend-cuda.cu:295-300
//   - the 12 kernels         backend-cuda.cu:302-434
//   - the step sequence      backend-cuda.cu:612-671 (alpha gating 622/656,
//                            pressure reset 644, dissipation 664-667)
// in two instances:
//   - Real = double: the accuracy oracle (every result states its error vs it);
//   - Real = float : the same sequence in FP32 with the multiply-add pairs
//     that the CUDA compiler contracts into fused multiply-adds written as
//     std::fma, parallelised with OpenMP; this is also the timed CPU
//     baseline (the reference has no CPU path of its own).
// Two iteration schemes: RBGS (the reference's in-place red-black Gauss-Seidel)
// and JACOBI (out-of-place sweeps), plus the FP64 relative Poisson residual.
//
// Pinning: tests/test_oracle_golden.py compares this file's FP32 instance with
// fixtures produced by the reference library itself (tests/golden/).

#include "stable-fluids-3d.h"

#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <new>
#include <type_traits>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace sfo {

struct Dims {
    int nx = 0, ny = 0, nz = 0;
    std::size_t n = 0;
};

// backend-cuda.cu:58-60 -- x-fastest linear index.
static inline std::size_t at(int x, int y, int z, const Dims& d) {
    return static_cast<std::size_t>(x) + static_cast<std::size_t>(d.nx) * (static_cast<std::size_t>(y) + static_cast<std::size_t>(d.ny) * static_cast<std::size_t>(z));
}

static inline int wrap(int c, int n) {
    c %= n;
    if (c < 0) c += n;
    return c;
}

static inline int clampi(int c, int lo, int hi) { return c < lo ? lo : (c > hi ? hi : c); }

// Multiply-add as the CUDA build evaluates it: fused (one rounding) in FP32,
// plain in FP64 where rounding is not the point.
template <class R>
static inline R mad(R a, R b, R c) {
    if constexpr (std::is_same_v<R, float>) return std::fma(a, b, c);
    else return a * b + c;
}

// a + (b - a) * t, backend-cuda.cu:232-238 / 282-288.
template <class R>
static inline R lerp(R a, R b, R t) { return mad(b - a, t, a); }

// Which evaluation order the sum of three products takes (divergence
// backend-cuda.cu:395, magnitude :433). The compiler's choice is not visible
// from the source; the golden fixtures select it (tests/test_oracle_golden.py).
enum SumOrder : int { SUM_FMA_OUTER_LAST = 0, SUM_FMA_INNER_LAST = 1, SUM_PLAIN = 2 };
static int g_sum_order = SUM_FMA_OUTER_LAST;

template <class R>
static inline R sum3_products(R a, R ka, R b, R kb, R c, R kc) {
    if constexpr (std::is_same_v<R, float>) {
        switch (g_sum_order) {
        case SUM_FMA_OUTER_LAST: return std::fma(c, kc, std::fma(a, ka, b * kb));
        case SUM_FMA_INNER_LAST: return std::fma(a, ka, std::fma(b, kb, c * kc));
        default: return (a * ka + b * kb) + c * kc;
        }
    } else {
        return a * ka + b * kb + c * kc;
    }
}

static inline bool flow_axis_periodic(const StableFluidsFlowBoundaryConfig& b, int axis) {
    const StableFluidsFlowBoundaryFaceDesc* f = &b.x_minus;
    return f[2 * axis].type == STABLE_FLUIDS_FLOW_BOUNDARY_PERIODIC && f[2 * axis + 1].type == STABLE_FLUIDS_FLOW_BOUNDARY_PERIODIC;
}
static inline bool scalar_axis_periodic(const StableFluidsScalarBoundaryConfig& b, int axis) {
    const StableFluidsScalarBoundaryFaceDesc* f = &b.x_minus;
    return f[2 * axis].type == STABLE_FLUIDS_SCALAR_BOUNDARY_PERIODIC && f[2 * axis + 1].type == STABLE_FLUIDS_SCALAR_BOUNDARY_PERIODIC;
}

// backend-cuda.cu:62-94 -- axes in order x, y, z: periodic wraps, zero-flux
// clamps and moves on, fixed-value returns the face value at once.
template <class R>
static R load_scalar(const R* f, int c0, int c1, int c2, const Dims& d, const StableFluidsScalarBoundaryConfig& b) {
    int c[3] = {c0, c1, c2};
    const int n[3] = {d.nx, d.ny, d.nz};
    const StableFluidsScalarBoundaryFaceDesc* faces = &b.x_minus;
    for (int a = 0; a < 3; ++a) {
        if (c[a] >= 0 && c[a] < n[a]) continue;
        const StableFluidsScalarBoundaryFaceDesc& face = faces[2 * a + (c[a] < 0 ? 0 : 1)];
        if (scalar_axis_periodic(b, a) && n[a] > 0) c[a] = wrap(c[a], n[a]);
        else if (face.type == STABLE_FLUIDS_SCALAR_BOUNDARY_ZERO_FLUX && n[a] > 0) c[a] = c[a] < 0 ? 0 : n[a] - 1;
        else return static_cast<R>(face.value);
    }
    return f[at(c[0], c[1], c[2], d)];
}

// backend-cuda.cu:96-128 -- periodic wraps, outflow is Dirichlet (face
// pressure), walls clamp (Neumann).
template <class R>
static R load_pressure(const R* f, int c0, int c1, int c2, const Dims& d, const StableFluidsFlowBoundaryConfig& b) {
    int c[3] = {c0, c1, c2};
    const int n[3] = {d.nx, d.ny, d.nz};
    const StableFluidsFlowBoundaryFaceDesc* faces = &b.x_minus;
    for (int a = 0; a < 3; ++a) {
        if (c[a] >= 0 && c[a] < n[a]) continue;
        const StableFluidsFlowBoundaryFaceDesc& face = faces[2 * a + (c[a] < 0 ? 0 : 1)];
        if (flow_axis_periodic(b, a) && n[a] > 0) c[a] = wrap(c[a], n[a]);
        else if (face.type == STABLE_FLUIDS_FLOW_BOUNDARY_OUTFLOW) return static_cast<R>(face.pressure);
        else c[a] = c[a] < 0 ? 0 : n[a] - 1;
    }
    return f[at(c[0], c[1], c[2], d)];
}

// backend-cuda.cu:130-189 -- periodic wraps and continues; any other face
// reads the interior at the face (all other axes clamped) and returns:
// outflow copies it, free-slip copies tangential components, everything else
// reflects about the prescribed wall velocity (2 v_wall - interior).
template <class R>
static R load_velocity(const R* f, int comp, int c0, int c1, int c2, const Dims& d, const StableFluidsFlowBoundaryConfig& b) {
    int c[3] = {c0, c1, c2};
    const int n[3] = {d.nx, d.ny, d.nz};
    const StableFluidsFlowBoundaryFaceDesc* faces = &b.x_minus;
    for (int a = 0; a < 3; ++a) {
        if (c[a] >= 0 && c[a] < n[a]) continue;
        const StableFluidsFlowBoundaryFaceDesc& face = faces[2 * a + (c[a] < 0 ? 0 : 1)];
        if (flow_axis_periodic(b, a) && n[a] > 0) {
            c[a] = wrap(c[a], n[a]);
            continue;
        }
        int q[3];
        for (int k = 0; k < 3; ++k) q[k] = clampi(c[k], 0, n[k] - 1);
        q[a] = c[a] < 0 ? 0 : n[a] - 1;
        const R interior = f[at(q[0], q[1], q[2], d)];
        const float prescribed = comp == 0 ? face.velocity_x : (comp == 1 ? face.velocity_y : face.velocity_z);
        if (face.type == STABLE_FLUIDS_FLOW_BOUNDARY_OUTFLOW) return interior;
        if (face.type == STABLE_FLUIDS_FLOW_BOUNDARY_FREE_SLIP_WALL && comp != a) return interior;
        return static_cast<R>(2.0f * prescribed) - interior;
    }
    return f[at(c[0], c[1], c[2], d)];
}

// backend-cuda.cu:195-206 / 245-256 -- periodic axes wrap the world position.
template <class R>
static inline R wrap_world(R p, R extent) {
    p = extent <= R(0) ? R(0) : std::fmod(p, extent);
    if (p < R(0)) p += extent;
    return p;
}

struct Corner {
    int x0, y0, z0;
};

// Trilinear sample (backend-cuda.cu:191-239 / 241-289) with a caller-supplied
// ghost-aware loader.
template <class R, class Load>
static R sample_trilinear(R x, R y, R z, R h, const Load& load) {
    const R gx = x / h - R(0.5);
    const R gy = y / h - R(0.5);
    const R gz = z / h - R(0.5);
    const int x0 = static_cast<int>(std::floor(gx));
    const int y0 = static_cast<int>(std::floor(gy));
    const int z0 = static_cast<int>(std::floor(gz));
    const R tx = gx - static_cast<R>(x0);
    const R ty = gy - static_cast<R>(y0);
    const R tz = gz - static_cast<R>(z0);
    const R c000 = load(x0, y0, z0), c100 = load(x0 + 1, y0, z0);
    const R c010 = load(x0, y0 + 1, z0), c110 = load(x0 + 1, y0 + 1, z0);
    const R c001 = load(x0, y0, z0 + 1), c101 = load(x0 + 1, y0, z0 + 1);
    const R c011 = load(x0, y0 + 1, z0 + 1), c111 = load(x0 + 1, y0 + 1, z0 + 1);
    const R c00 = lerp(c000, c100, tx);
    const R c10 = lerp(c010, c110, tx);
    const R c01 = lerp(c001, c101, tx);
    const R c11 = lerp(c011, c111, tx);
    const R c0 = lerp(c00, c10, ty);
    const R c1 = lerp(c01, c11, ty);
    return lerp(c0, c1, tz);
}

template <class R>
struct Flow {
    const StableFluidsFlowBoundaryConfig* bc;
    Dims d;
    R h;
};

template <class R>
static R sample_velocity(const R* f, int comp, R x, R y, R z, const Flow<R>& fl) {
    const R ex = static_cast<R>(fl.d.nx) * fl.h, ey = static_cast<R>(fl.d.ny) * fl.h, ez = static_cast<R>(fl.d.nz) * fl.h;
    if (flow_axis_periodic(*fl.bc, 0)) x = wrap_world(x, ex);
    if (flow_axis_periodic(*fl.bc, 1)) y = wrap_world(y, ey);
    if (flow_axis_periodic(*fl.bc, 2)) z = wrap_world(z, ez);
    return sample_trilinear<R>(x, y, z, fl.h, [&](int a, int b, int c) { return load_velocity(f, comp, a, b, c, fl.d, *fl.bc); });
}

template <class R>
static R sample_scalar(const R* f, R x, R y, R z, R h, const Dims& d, const StableFluidsScalarBoundaryConfig& bc) {
    const R ex = static_cast<R>(d.nx) * h, ey = static_cast<R>(d.ny) * h, ez = static_cast<R>(d.nz) * h;
    if (scalar_axis_periodic(bc, 0)) x = wrap_world(x, ex);
    if (scalar_axis_periodic(bc, 1)) y = wrap_world(y, ey);
    if (scalar_axis_periodic(bc, 2)) z = wrap_world(z, ez);
    return sample_trilinear<R>(x, y, z, h, [&](int a, int b, int c) { return load_scalar(f, a, b, c, d, bc); });
}

// backend-cuda.cu:295-300 -- midpoint RK2 back-trace in world units.
template <class R>
static void trace_rk2(R px, R py, R pz, const R* vx, const R* vy, const R* vz, R dt, const Flow<R>& fl, R out[3]) {
    const R v0x = sample_velocity(vx, 0, px, py, pz, fl);
    const R v0y = sample_velocity(vy, 1, px, py, pz, fl);
    const R v0z = sample_velocity(vz, 2, px, py, pz, fl);
    const R half_dt = R(0.5) * dt;
    const R mx = mad(-half_dt, v0x, px), my = mad(-half_dt, v0y, py), mz = mad(-half_dt, v0z, pz);
    const R v1x = sample_velocity(vx, 0, mx, my, mz, fl);
    const R v1y = sample_velocity(vy, 1, mx, my, mz, fl);
    const R v1z = sample_velocity(vz, 2, mx, my, mz, fl);
    out[0] = mad(-dt, v1x, px);
    out[1] = mad(-dt, v1y, py);
    out[2] = mad(-dt, v1z, pz);
}

enum Scheme : int { RBGS = 0, JACOBI = 1 };

struct ScalarDesc {
    StableFluidsScalarFieldDesc desc;
};

template <class R>
struct Sim {
    StableFluidsSimulationConfig cfg{};
    Dims d;
    int scheme = RBGS;
    int warm_previous = 0;
    std::vector<R> vel[3], tmp[3], pressure, divergence, magnitude, scratch;
    struct Scalar {
        StableFluidsScalarFieldDesc desc;
        std::vector<R> data, temp, source;
    };
    struct Vector {
        StableFluidsVectorFieldDesc desc;
        std::vector<R> data[3];
    };
    std::vector<Scalar> scalars;
    std::vector<Vector> vectors;
    // residual-driven pressure solve (0 = fixed iteration count)
    double tolerance = 0.0;
    int max_iterations = 0, check_interval = 1;
    int compute_residual = 0;
    // statistics of the last step
    double last_rel_residual = -1.0, last_rhs_norm = 0.0;
    int last_iterations = 0, last_hit_cap = 0;

    R h() const { return static_cast<R>(cfg.cell_size); }
    R dt() const { return static_cast<R>(cfg.dt); }

    void init(const StableFluidsContextCreateDesc& desc) {
        cfg = desc.config;
        d.nx = cfg.nx;
        d.ny = cfg.ny;
        d.nz = cfg.nz;
        d.n = static_cast<std::size_t>(d.nx) * d.ny * d.nz;
        for (int c = 0; c < 3; ++c) {
            vel[c].assign(d.n, R(0));
            tmp[c].assign(d.n, R(0));
        }
        pressure.assign(d.n, R(0));
        divergence.assign(d.n, R(0));
        magnitude.assign(d.n, R(0));
        scratch.assign(d.n, R(0));
        for (uint32_t i = 0; i < desc.scalar_field_count; ++i) {
            Scalar s;
            s.desc = desc.scalar_fields[i];
            s.data.assign(d.n, static_cast<R>(s.desc.initial_value));
            s.temp.assign(d.n, static_cast<R>(s.desc.initial_value));
            s.source.assign(d.n, R(0));
            scalars.push_back(std::move(s));
        }
        for (uint32_t i = 0; i < desc.vector_field_count; ++i) {
            Vector v;
            v.desc = desc.vector_fields[i];
            v.data[0].assign(d.n, static_cast<R>(v.desc.initial_value_x));
            v.data[1].assign(d.n, static_cast<R>(v.desc.initial_value_y));
            v.data[2].assign(d.n, static_cast<R>(v.desc.initial_value_z));
            vectors.push_back(std::move(v));
        }
    }

    // ---- per-stage restatements -------------------------------------------

    // backend-cuda.cu:310-319 / 612-615
    void add_forces() {
        const R dt_ = dt();
        for (auto& v : vectors) {
            if (v.desc.usage != STABLE_FLUIDS_VECTOR_FIELD_FORCE) continue;
            for (int c = 0; c < 3; ++c) {
                R* u = vel[c].data();
                const R* f = v.data[c].data();
#pragma omp parallel for schedule(static)
                for (long long i = 0; i < static_cast<long long>(d.n); ++i) u[i] = mad(dt_, f[i], u[i]);
            }
        }
    }

    // backend-cuda.cu:330-340 / 617-619 (the trace is recomputed per component
    // upstream; it is deterministic, so tracing once per cell is identical).
    void advect_velocity() {
        const Flow<R> fl{&cfg.flow_boundary, d, h()};
        const R dt_ = dt(), h_ = h();
#pragma omp parallel for schedule(static)
        for (int z = 0; z < d.nz; ++z)
            for (int y = 0; y < d.ny; ++y)
                for (int x = 0; x < d.nx; ++x) {
                    const R px = (static_cast<R>(x) + R(0.5)) * h_, py = (static_cast<R>(y) + R(0.5)) * h_, pz = (static_cast<R>(z) + R(0.5)) * h_;
                    R t[3];
                    trace_rk2(px, py, pz, vel[0].data(), vel[1].data(), vel[2].data(), dt_, fl, t);
                    const std::size_t i = at(x, y, z, d);
                    for (int c = 0; c < 3; ++c) tmp[c][i] = sample_velocity(vel[c].data(), c, t[0], t[1], t[2], fl);
                }
    }

    // backend-cuda.cu:342-352 / 654 (scalar sampled with its own boundary,
    // trace with the flow boundary, projected velocity).
    void advect_scalar(Scalar& s) {
        const Flow<R> fl{&cfg.flow_boundary, d, h()};
        const R dt_ = dt(), h_ = h();
#pragma omp parallel for schedule(static)
        for (int z = 0; z < d.nz; ++z)
            for (int y = 0; y < d.ny; ++y)
                for (int x = 0; x < d.nx; ++x) {
                    const R px = (static_cast<R>(x) + R(0.5)) * h_, py = (static_cast<R>(y) + R(0.5)) * h_, pz = (static_cast<R>(z) + R(0.5)) * h_;
                    R t[3];
                    trace_rk2(px, py, pz, vel[0].data(), vel[1].data(), vel[2].data(), dt_, fl, t);
                    s.temp[at(x, y, z, d)] = sample_scalar(s.data.data(), t[0], t[1], t[2], h_, d, s.desc.boundary);
                }
    }

    // One colour of a diffusion RBGS iteration, backend-cuda.cu:354-375:
    // x = (b + alpha * sum6(x)) / (1 + 6 alpha), neighbour order
    // x-, x+, y-, y+, z-, z+; JACOBI (parity < 0) reads src_x, writes dst_x
    // and multiplies by the rounded reciprocal instead of dividing (the
    // library's Jacobi arithmetic; the reference has no Jacobi scheme).
    template <class Load>
    void diffuse_pass(R* dst, const R* srcx, const R* b, R alpha, int parity, const Load& load) {
        const R denom = mad(R(6), alpha, R(1));
        const R inv = R(1) / denom;
#pragma omp parallel for schedule(static)
        for (int z = 0; z < d.nz; ++z)
            for (int y = 0; y < d.ny; ++y)
                for (int x = 0; x < d.nx; ++x) {
                    if (parity >= 0 && ((x + y + z) & 1) != parity) continue;
                    const R nb = load(srcx, x - 1, y, z) + load(srcx, x + 1, y, z) + load(srcx, x, y - 1, z) + load(srcx, x, y + 1, z) + load(srcx, x, y, z - 1) + load(srcx, x, y, z + 1);
                    const std::size_t i = at(x, y, z, d);
                    dst[i] = parity >= 0 ? mad(alpha, nb, b[i]) / denom : mad(alpha, nb, b[i]) * inv;
                }
    }

    template <class Load>
    void diffuse(std::vector<R>& x, const std::vector<R>& b, R alpha, const Load& load) {
        for (int it = 0; it < cfg.diffuse_iterations; ++it) {
            if (scheme == RBGS) {
                diffuse_pass(x.data(), x.data(), b.data(), alpha, 0, load);
                diffuse_pass(x.data(), x.data(), b.data(), alpha, 1, load);
            } else {
                diffuse_pass(scratch.data(), x.data(), b.data(), alpha, -1, load);
                x.swap(scratch);
            }
        }
    }

    // backend-cuda.cu:386-396 -- central differences with velocity ghosts.
    void compute_divergence() {
        const Flow<R> fl{&cfg.flow_boundary, d, h()};
        const R inv2h = R(0.5) / h();
#pragma omp parallel for schedule(static)
        for (int z = 0; z < d.nz; ++z)
            for (int y = 0; y < d.ny; ++y)
                for (int x = 0; x < d.nx; ++x) {
                    const R dx = load_velocity(vel[0].data(), 0, x + 1, y, z, d, *fl.bc) - load_velocity(vel[0].data(), 0, x - 1, y, z, d, *fl.bc);
                    const R dy = load_velocity(vel[1].data(), 1, x, y + 1, z, d, *fl.bc) - load_velocity(vel[1].data(), 1, x, y - 1, z, d, *fl.bc);
                    const R dz = load_velocity(vel[2].data(), 2, x, y, z + 1, d, *fl.bc) - load_velocity(vel[2].data(), 2, x, y, z - 1, d, *fl.bc);
                    divergence[at(x, y, z, d)] = sum3_products(dx, inv2h, dy, inv2h, dz, inv2h);
                }
    }

    // backend-cuda.cu:398-407 -- p = (sum6(p) - h^2 div) / 6; JACOBI
    // (parity < 0) multiplies by the rounded reciprocal RN(1/6) instead.
    void pressure_pass(R* dst, const R* src, R h2, int parity) {
        const auto& bc = cfg.flow_boundary;
        const R inv6 = R(1) / R(6);
#pragma omp parallel for schedule(static)
        for (int z = 0; z < d.nz; ++z)
            for (int y = 0; y < d.ny; ++y)
                for (int x = 0; x < d.nx; ++x) {
                    if (parity >= 0 && ((x + y + z) & 1) != parity) continue;
                    const R nb = load_pressure(src, x - 1, y, z, d, bc) + load_pressure(src, x + 1, y, z, d, bc) + load_pressure(src, x, y - 1, z, d, bc) + load_pressure(src, x, y + 1, z, d, bc) + load_pressure(src, x, y, z - 1, d, bc)
                               + load_pressure(src, x, y, z + 1, d, bc);
                    const std::size_t i = at(x, y, z, d);
                    dst[i] = parity >= 0 ? mad(-h2, divergence[i], nb) / R(6) : mad(-h2, divergence[i], nb) * inv6;
                }
    }

    void pressure_iteration(R h2) {
        if (scheme == RBGS) {
            pressure_pass(pressure.data(), pressure.data(), h2, 0);
            pressure_pass(pressure.data(), pressure.data(), h2, 1);
        } else {
            pressure_pass(scratch.data(), pressure.data(), h2, -1);
            pressure.swap(scratch);
        }
    }

    bool pressure_singular() const {
        const StableFluidsFlowBoundaryFaceDesc* f = &cfg.flow_boundary.x_minus;
        for (int k = 0; k < 6; ++k)
            if (f[k].type == STABLE_FLUIDS_FLOW_BOUNDARY_OUTFLOW) return false;
        return true;
    }

    // FP64 relative residual of the pressure system A p = b, b = h^2 div,
    // A p = sum6(p) - 6 p with the pressure ghost rules; b's mean is removed
    // when A is singular (no outflow face).
    double rel_residual(double* rhs_norm_out) const {
        const auto& bc = cfg.flow_boundary;
        const double h2 = static_cast<double>(static_cast<float>(cfg.cell_size * cfg.cell_size));
        double se = 0, se2 = 0, sb = 0, sb2 = 0;
        const R* p = pressure.data();
#pragma omp parallel for schedule(static) reduction(+ : se, se2, sb, sb2)
        for (int z = 0; z < d.nz; ++z)
            for (int y = 0; y < d.ny; ++y)
                for (int x = 0; x < d.nx; ++x) {
                    const double nb = static_cast<double>(load_pressure(p, x - 1, y, z, d, bc)) + static_cast<double>(load_pressure(p, x + 1, y, z, d, bc)) + static_cast<double>(load_pressure(p, x, y - 1, z, d, bc)) + static_cast<double>(load_pressure(p, x, y + 1, z, d, bc))
                                    + static_cast<double>(load_pressure(p, x, y, z - 1, d, bc)) + static_cast<double>(load_pressure(p, x, y, z + 1, d, bc));
                    const std::size_t i = at(x, y, z, d);
                    const double b = h2 * static_cast<double>(divergence[i]);
                    const double e = b - (nb - 6.0 * static_cast<double>(p[i]));
                    se += e;
                    se2 += e * e;
                    sb += b;
                    sb2 += b * b;
                }
        const double n = static_cast<double>(d.n);
        double r2 = se2, b2 = sb2;
        if (pressure_singular()) {
            const double mb = sb / n;
            r2 = se2 - 2.0 * mb * se + n * mb * mb;
            b2 = sb2 - n * mb * mb;
        }
        if (r2 < 0) r2 = 0;
        if (b2 < 0) b2 = 0;
        if (rhs_norm_out) *rhs_norm_out = std::sqrt(b2);
        return b2 > 0 ? std::sqrt(r2) / std::sqrt(b2) : 0.0;
    }

    // backend-cuda.cu:409-422 -- u -= central gradient of p (in place).
    void project() {
        const auto& bc = cfg.flow_boundary;
        const R inv2h = R(0.5) / h();
        const R* p = pressure.data();
#pragma omp parallel for schedule(static)
        for (int z = 0; z < d.nz; ++z)
            for (int y = 0; y < d.ny; ++y)
                for (int x = 0; x < d.nx; ++x) {
                    const std::size_t i = at(x, y, z, d);
                    const R gx = load_pressure(p, x + 1, y, z, d, bc) - load_pressure(p, x - 1, y, z, d, bc);
                    const R gy = load_pressure(p, x, y + 1, z, d, bc) - load_pressure(p, x, y - 1, z, d, bc);
                    const R gz = load_pressure(p, x, y, z + 1, d, bc) - load_pressure(p, x, y, z - 1, d, bc);
                    vel[0][i] = mad(-gx, inv2h, vel[0][i]);
                    vel[1][i] = mad(-gy, inv2h, vel[1][i]);
                    vel[2][i] = mad(-gz, inv2h, vel[2][i]);
                }
    }

    // backend-cuda.cu:424-434
    void velocity_magnitude() {
#pragma omp parallel for schedule(static)
        for (long long i = 0; i < static_cast<long long>(d.n); ++i) {
            const R a = vel[0][i], b = vel[1][i], c = vel[2][i];
            magnitude[i] = std::sqrt(sum3_products(a, a, b, b, c, c));
        }
    }

    // ---- the step, backend-cuda.cu:612-671 --------------------------------
    void step() {
        const float hf = cfg.cell_size;
        add_forces();
        const float alpha_v_f = cfg.dt * cfg.viscosity / (hf * hf);  // :622 (host FP32)
        const R alpha_v = static_cast<R>(alpha_v_f);
        // The advected velocity only survives when diffusion runs (:623-626).
        if (alpha_v_f > 0.0f) {
            advect_velocity();
            for (int c = 0; c < 3; ++c) vel[c] = tmp[c];
            for (int c = 0; c < 3; ++c) {
                const auto& bc = cfg.flow_boundary;
                diffuse(vel[c], tmp[c], alpha_v, [&, c](const R* f, int x, int y, int z) { return load_velocity(f, c, x, y, z, d, bc); });
            }
        }
        compute_divergence();
        if (!warm_previous) std::fill(pressure.begin(), pressure.end(), R(0));  // :644
        const float h2f = hf * hf;  // :645
        const R h2 = static_cast<R>(h2f);
        last_hit_cap = 0;
        if (tolerance > 0.0) {
            int it = 0;
            double rr = rel_residual(&last_rhs_norm);
            while (rr > tolerance && it < max_iterations) {
                const int k = std::min(check_interval, max_iterations - it);
                if (scheme == JACOBI) {
                    // the library measures the residual inside the interval's
                    // last sweep, i.e. of the iterate one sweep before
                    for (int j = 0; j + 1 < k; ++j) pressure_iteration(h2);
                    rr = rel_residual(&last_rhs_norm);
                    pressure_iteration(h2);
                } else {
                    for (int j = 0; j < k; ++j) pressure_iteration(h2);
                    rr = rel_residual(&last_rhs_norm);
                }
                it += k;
            }
            last_iterations = it;
            last_rel_residual = rr;
            last_hit_cap = rr > tolerance ? 1 : 0;
        } else {
            for (int it = 0; it < cfg.pressure_iterations; ++it) pressure_iteration(h2);
            last_iterations = cfg.pressure_iterations;
            last_rel_residual = compute_residual ? rel_residual(&last_rhs_norm) : -1.0;
        }
        project();
        for (auto& s : scalars) {
            const R dt_ = dt();
            {
                R* q = s.data.data();
                const R* src = s.source.data();
#pragma omp parallel for schedule(static)
                for (long long i = 0; i < static_cast<long long>(d.n); ++i) q[i] = mad(dt_, src[i], q[i]);  // :321-328
            }
            const float alpha_s_f = cfg.dt * s.desc.diffusion / (hf * hf);  // :656
            if (alpha_s_f > 0.0f) {
                advect_scalar(s);
                s.data = s.temp;
                const auto& bc = s.desc.boundary;
                diffuse(s.data, s.temp, static_cast<R>(alpha_s_f), [&](const R* f, int x, int y, int z) { return load_scalar(f, x, y, z, d, bc); });
            }
            if (s.desc.dissipation > 0.0f) {
                const float factor = 1.0f / (1.0f + cfg.dt * s.desc.dissipation);  // :665 (host FP32)
                const R fr = static_cast<R>(factor);
                for (auto& q : s.data) q = q * fr;  // :377-384
            }
        }
        compute_divergence();  // :670 (post-projection)
        velocity_magnitude();  // :671
    }
};

struct Handle {
    int precision = 64;
    std::unique_ptr<Sim<double>> d64;
    std::unique_ptr<Sim<float>> f32;
};

template <class R, class F>
static int with_sim(Handle* h, F&& f) {
    (void)sizeof(R);
    if (h->precision == 64) return f(*h->d64);
    return f(*h->f32);
}

}  // namespace sfo

extern "C" {

// Create an oracle simulation. precision: 32 or 64. scheme: 0 RBGS, 1 JACOBI.
int sfo_create(const StableFluidsContextCreateDesc* desc, int precision, int scheme, void** out) {
    if (!desc || !out || (precision != 32 && precision != 64)) return 2;
    const auto& c = desc->config;
    if (c.nx <= 0 || c.ny <= 0 || c.nz <= 0) return 2;
    auto* h = new (std::nothrow) sfo::Handle;
    if (!h) return 1;
    h->precision = precision;
    if (precision == 64) {
        h->d64 = std::make_unique<sfo::Sim<double>>();
        h->d64->scheme = scheme;
        h->d64->init(*desc);
    } else {
        h->f32 = std::make_unique<sfo::Sim<float>>();
        h->f32->scheme = scheme;
        h->f32->init(*desc);
    }
    *out = h;
    return 0;
}

void sfo_destroy(void* handle) { delete static_cast<sfo::Handle*>(handle); }

// Residual-driven pressure solve (tolerance > 0) or fixed count (tolerance 0);
// warm_previous keeps the last pressure as the initial guess.
int sfo_set_solver(void* handle, double tolerance, int max_iterations, int check_interval, int warm_previous, int compute_residual) {
    auto* h = static_cast<sfo::Handle*>(handle);
    auto apply = [&](auto& s) {
        s.tolerance = tolerance;
        s.max_iterations = max_iterations;
        s.check_interval = check_interval < 1 ? 1 : check_interval;
        s.warm_previous = warm_previous;
        s.compute_residual = compute_residual;
        return 0;
    };
    return h->precision == 64 ? apply(*h->d64) : apply(*h->f32);
}

void sfo_set_sum_order(int order) { sfo::g_sum_order = order; }

int sfo_set_threads(int threads) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
    return omp_get_max_threads();
#else
    (void)threads;
    return 1;
#endif
}

// kind: 0 scalar data, 1 scalar source, 2 vector field, 3 velocity,
// 4 magnitude, 5 pressure, 6 divergence, 7 scalar temp, 8 velocity temp.
int sfo_set_field(void* handle, int kind, uint32_t field, int component, const float* values) {
    auto* h = static_cast<sfo::Handle*>(handle);
    auto apply = [&](auto& s) -> int {
        using R = typename std::remove_reference_t<decltype(s.pressure)>::value_type;
        std::vector<R>* dst = nullptr;
        if (kind == 0 || kind == 1) {
            if (field == 0 || field > s.scalars.size()) return 2;
            dst = kind == 0 ? &s.scalars[field - 1].data : &s.scalars[field - 1].source;
        } else if (kind == 2) {
            if (field == 0 || field > s.vectors.size() || component < 0 || component > 2) return 2;
            dst = &s.vectors[field - 1].data[component];
        } else if (kind == 3) {
            if (component < 0 || component > 2) return 2;
            dst = &s.vel[component];
        } else if (kind == 5) {
            dst = &s.pressure;
        } else {
            return 2;
        }
        for (std::size_t i = 0; i < s.d.n; ++i) (*dst)[i] = values ? static_cast<R>(values[i]) : R(0);
        return 0;
    };
    return h->precision == 64 ? apply(*h->d64) : apply(*h->f32);
}

int sfo_get_field(void* handle, int kind, uint32_t field, int component, double* out) {
    auto* h = static_cast<sfo::Handle*>(handle);
    auto apply = [&](auto& s) -> int {
        using R = typename std::remove_reference_t<decltype(s.pressure)>::value_type;
        const std::vector<R>* src = nullptr;
        switch (kind) {
        case 0:
        case 1:
        case 7:
            if (field == 0 || field > s.scalars.size()) return 2;
            src = kind == 0 ? &s.scalars[field - 1].data : (kind == 1 ? &s.scalars[field - 1].source : &s.scalars[field - 1].temp);
            break;
        case 2:
            if (field == 0 || field > s.vectors.size() || component < 0 || component > 2) return 2;
            src = &s.vectors[field - 1].data[component];
            break;
        case 3:
        case 8:
            if (component < 0 || component > 2) return 2;
            src = kind == 3 ? &s.vel[component] : &s.tmp[component];
            break;
        case 4: src = &s.magnitude; break;
        case 5: src = &s.pressure; break;
        case 6: src = &s.divergence; break;
        default: return 2;
        }
        for (std::size_t i = 0; i < s.d.n; ++i) out[i] = static_cast<double>((*src)[i]);
        return 0;
    };
    return h->precision == 64 ? apply(*h->d64) : apply(*h->f32);
}

int sfo_step(void* handle, int steps) {
    auto* h = static_cast<sfo::Handle*>(handle);
    for (int k = 0; k < steps; ++k) {
        if (h->precision == 64) h->d64->step();
        else h->f32->step();
    }
    return 0;
}

// Statistics of the last step: rel_res (or -1), ||b||, iterations, cap flag.
int sfo_get_stats(void* handle, double* rel_residual, double* rhs_norm, int* iterations, int* hit_cap) {
    auto* h = static_cast<sfo::Handle*>(handle);
    auto apply = [&](auto& s) {
        if (rel_residual) *rel_residual = s.last_rel_residual;
        if (rhs_norm) *rhs_norm = s.last_rhs_norm;
        if (iterations) *iterations = s.last_iterations;
        if (hit_cap) *hit_cap = s.last_hit_cap;
        return 0;
    };
    return h->precision == 64 ? apply(*h->d64) : apply(*h->f32);
}

// The FP64 residual of the current pressure/divergence pair.
double sfo_rel_residual(void* handle, double* rhs_norm) {
    auto* h = static_cast<sfo::Handle*>(handle);
    return h->precision == 64 ? h->d64->rel_residual(rhs_norm) : h->f32->rel_residual(rhs_norm);
}

}  // extern "C"
