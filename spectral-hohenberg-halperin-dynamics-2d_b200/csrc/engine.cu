// Host side of the step engine: plans, device buffers, launch sequence and
// the C ABI declared in include/shhd_b200.h.
//
// One engine = one configuration (grid, mode, models) and `batch` members.
// A step of all members is, per right-hand-side stage, one row_pass launch
// and one col_forward launch (which also produces the next stage's column
// inverse); each step call starts with one col_inverse launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/shhd_b200.h"
#include "step_kernels.cuh"
#include "step_kernels_fixed.cuh"
#include "step_kernels_pair.cuh"
#include "step_reg.h"

using namespace shhd;

namespace {

thread_local std::string g_last_error;

struct Failure : std::runtime_error {
    int code;
    Failure(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw Failure(SHHD_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

template <typename F>
int guarded(F&& f) {
    try {
        f();
        return SHHD_OK;
    } catch (const Failure& e) {
        g_last_error = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        g_last_error = "host allocation failed";
        return SHHD_ENOMEM;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return SHHD_EINVAL;
    }
}

// ---------------------------------------------------------------------------
// FFT plans
// ---------------------------------------------------------------------------
FftPlan make_fft_plan(int n) {
    FftPlan p{};
    p.n = n;
    int m = n;
    std::vector<int> rad;
    for (int r : {8, 4, 2}) while (m % r == 0) { rad.push_back(r); m /= r; }
    while (m % 3 == 0) { rad.push_back(3); m /= 3; }
    while (m % 5 == 0) { rad.push_back(5); m /= 5; }
    if (m != 1)
        throw Failure(SHHD_EUNSUPPORTED, "compute grid size " + std::to_string(n) + " has a prime factor other than 2, 3, 5");
    if (static_cast<int>(rad.size()) > kMaxStages) throw Failure(SHHD_EUNSUPPORTED, "compute grid size too large");
    p.nstages = static_cast<int>(rad.size());
    int span = 1;
    for (int s = 0; s < p.nstages; ++s) {
        p.radix[s] = rad[s];
        p.span[s] = span;
        p.twstride[s] = n / (span * rad[s]);
        p.div_nr[s] = make_fastdiv(static_cast<uint32_t>(n / rad[s]));
        p.div_p[s] = make_fastdiv(static_cast<uint32_t>(span));
        span *= rad[s];
    }
    p.tw_hi_count = (n + kTwLo - 1) / kTwLo;
    return p;
}

// shared-memory swizzle mask: `slots` complex values make one bank wavefront
// (16 for float2, 8 for double2) and `width` lines are interleaved; the mask
// must keep sw() inside aligned blocks the line length is a multiple of.
int swizzle_mask(int n, int slots, int width) {
    int m = std::max(1, slots / std::max(1, width)) - 1;
    while (m > 0 && n % (m + 1) != 0) m >>= 1;
    return m;
}

template <typename T>
std::vector<cplx<T>> twiddle_table(int n) {
    const int hi = (n + kTwLo - 1) / kTwLo;
    std::vector<cplx<T>> t(kTwLo + hi);
    for (int j = 0; j < kTwLo; ++j) {
        const double a = -2.0 * M_PI * static_cast<double>(j) / n;
        t[j].x = static_cast<T>(std::cos(a));
        t[j].y = static_cast<T>(std::sin(a));
    }
    for (int i = 0; i < hi; ++i) {
        const double a = -2.0 * M_PI * static_cast<double>((static_cast<long>(i) * kTwLo) % n) / n;
        t[kTwLo + i].x = static_cast<T>(std::cos(a));
        t[kTwLo + i].y = static_cast<T>(std::sin(a));
    }
    return t;
}

// per-stage twiddle rows of a compile-time plan (forward sign)
template <typename T>
std::vector<cplx<T>> stage_table(int n) {
    const CPlan c = make_cplan(n);
    std::vector<cplx<T>> t(std::max(c.twsz, 2));
    for (auto& z : t) { z.x = 0; z.y = 0; }
    for (int s = 0; s < c.ns; ++s) {
        const int R = c.r[s], p = c.p[s];
        if (p == 1) continue;
        for (int k = 0; k < p; ++k)
            for (int q = 1; q < R; ++q) {
                const double a = -2.0 * M_PI * static_cast<double>(q) * k / (static_cast<double>(p) * R);
                cplx<T>& z = t[c.twoff[s] + k * tw_row(R) + (q - 1)];
                z.x = static_cast<T>(std::cos(a));
                z.y = static_cast<T>(std::sin(a));
            }
    }
    return t;
}

int fixed_of(int n) { return is_fixed_size(n) ? n : 0; }

// call f(std::integral_constant<int, N>) for the compile-time size N (0 = runtime plan)
template <typename F>
void with_size(int n, F&& f) {
    switch (fixed_of(n)) {
        case 96: f(std::integral_constant<int, 96>{}); break;
        case 192: f(std::integral_constant<int, 192>{}); break;
        case 384: f(std::integral_constant<int, 384>{}); break;
        case 768: f(std::integral_constant<int, 768>{}); break;
        case 1536: f(std::integral_constant<int, 1536>{}); break;
        case 3072: f(std::integral_constant<int, 3072>{}); break;
        case 6144: f(std::integral_constant<int, 6144>{}); break;
        default: f(std::integral_constant<int, 0>{}); break;
    }
}

// call f(std::integral_constant<int, N>) for a pair-path size N (0 = none)
template <typename F>
void with_pair_size(int n, F&& f) {
    switch (n) {
        case 96: f(std::integral_constant<int, 96>{}); break;
        case 192: f(std::integral_constant<int, 192>{}); break;
        case 384: f(std::integral_constant<int, 384>{}); break;
        case 768: f(std::integral_constant<int, 768>{}); break;
        case 1536: f(std::integral_constant<int, 1536>{}); break;
        default: f(std::integral_constant<int, 0>{}); break;
    }
}

}  // namespace

namespace shhd_internal {
void set_last_error(const std::string& msg) { g_last_error = msg; }
}  // namespace shhd_internal

// ---------------------------------------------------------------------------
// engine
// ---------------------------------------------------------------------------
// Transforms of the physical-space measures: runtime-plan column and row transforms of one member,
// independent of the step's kernel family, with their own twiddle tables and scratch (built on first use).
struct MeasurePlan {
    bool ready = false;
    StepPlan P{};                 // geometry, physics and transforms; inputs are set per term
    void* tw_x = nullptr;
    void* tw_y = nullptr;
    void* i1 = nullptr;           // up to 3 x-spectral planes of one member
    void* member = nullptr;       // one always-active MemberInfo
    double* scratch = nullptr;    // partial sums, then the summed values
    size_t scratch_doubles = 0;
    double* profile = nullptr;    // profile partial rows [pairs][npx] and the result (allocated on first use)
    int* flag = nullptr;
    double2* line = nullptr;      // one spectral line of a profile sample
    size_t smem_col = 0, smem_row = 0;
};

struct shhd_engine {
    shhd_config cfg{};
    StepPlan P{};
    int fp32 = 0;
    size_t csize = 16;            // bytes per complex element
    cudaStream_t stream = nullptr;
    int device = 0;

    void* u = nullptr;
    void* s1 = nullptr;
    void* s2 = nullptr;
    void* i1 = nullptr;
    void* i2 = nullptr;
    void* ext_a = nullptr;
    void* ext_b = nullptr;
    void* det = nullptr;
    void* tw_x = nullptr;
    void* tw_y = nullptr;
    double* rho0_dev = nullptr;
    double2* k0_u = nullptr;         // FP64 k = 0 modes [member][field] of u, s1, s2 (FP32 engines)
    double2* k0_s1 = nullptr;
    double2* k0_s2 = nullptr;
    double* sk_dev = nullptr;        // FP64 structure-factor accumulator [Hx * Ky] (allocated on first use)
    double* l2_dev = nullptr;        // FP64 spectral L2 sums [field][2] (allocated on first use)
    // Yokota-Green-Kubo taps (FP64): selected modes, step flux, block integrals, sums [member][tau][mode]
    bool fline_on[2] = {false, false};
    FluxLineArgs fline[2]{};         // the step's flux buffer along the ky = 0 row / kx = 0 column (allocated on enable)
    bool flux0_on = false;
    Flux0Args flux0{};               // k = 0 fluxes of the last step [member][3 + 2 nop] (allocated on enable)
    bool gk_on = false;
    GkArgs gk{};
    std::vector<int2> gk_modes;
    std::vector<int64_t> gk_sample_base;
    int64_t sk_count = 0;
    int sk_field = -1;
    int* err_dev = nullptr;
    MemberInfo* members_dev = nullptr;
    std::vector<MemberInfo> members;
    bool members_dirty = true;
    int* static_dev = nullptr;
    int n_static = 0;

    size_t state_elems = 0;       // complex per member
    size_t i1_elems = 0, i2_elems = 0;
    int npos = 16;
    bool col_fixed = false;       // compile-time column kernels (group per column)
    bool row_fixed = false;       // compile-time row kernel (group per line)
    int row_nt = 256;             // its threads per block (512: two line groups, for lines of 48 KB or more)
    bool pair_path = false;       // FP32 pair-line kernels (compile-time sizes up to 1536)
    bool reg_row = false;         // register-resident row pass on 1536-point rows (pair-line layout)
    int family_override = -1;     // -1 choose (1 where valid, else 0), 0 never the pair-line kernels, 1 pair-line where valid,
                                  // 2 pair-line with the register-resident row pass where valid,
                                  // 3 pair-line with the split row pass where valid,
                                  // 4 pair-line with the two-pair row pass where valid
    int row_blocks = 0;           // pair-line row pass compiled for 2 or 3 blocks per SM (0: by its shared memory)
    int col_blocks = 0;           // pair-line column forward on >= 384-point columns for 3 or 4 blocks per SM (0: by rule)
    void* tw_reg = nullptr;       // twiddles of the register-resident transforms (FP32 engines with 1536-point rows)
    bool split_row = false;       // pair-line row pass split in two kernels over a physical-row buffer (family 3)
    bool dual_row = false;        // pair-line row pass over two output pairs at a time (family 4)
    size_t smem_dual = 0;
    void* phys = nullptr;         // that buffer, [member][row pair][input pair-line][npx] pair elements
    size_t phys_bytes = 0;
    size_t smem_rrow = 0;
    size_t tw_bytes = 0;
    size_t smem_col_inv = 0;
    size_t smem_col = 0, smem_row = 0;
    int n_evolved = 0;
    bool need_rho0 = false;
    std::vector<double> rho0_candidate;
    std::vector<int> rho0_cached;
    std::vector<double> rho0_value;
    size_t device_bytes = 0;

    int64_t step_index = 0;
    double time = 0.0;

    void* ref_stage = nullptr;       // one member's reference-layout state (FP64) on the device
    int* flag_dev = nullptr;
    MeasurePlan meas;
    double* ic_scratch = nullptr;    // random-vorticity norm [0] and block partial sums [1..]
    size_t ic_scratch_bytes = 0;
    unsigned long long* step_dev = nullptr;  // step index at the start of the current call

    // captured step graphs: one call of `size` steps each, for the chunk and every power of two
    // below it (a call is replayed as a sum of those), captured on first use
    struct CachedGraph {
        cudaGraphExec_t exec = nullptr;
        int64_t launches[4] = {0, 0, 0, 0};
        double bytes[4] = {0, 0, 0, 0};
    };
    int graph_chunk = 0;
    std::map<int, CachedGraph> graphs;

    // per-kernel statistics: 0 col_inverse, 1 row_pass, 2 col_forward, 3 other
    bool profiling = false;
    struct Pending { int kind; cudaEvent_t a, b; };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> event_pool;
    double kernel_ms[4] = {0, 0, 0, 0};
    int64_t kernel_launches[4] = {0, 0, 0, 0};
    double kernel_bytes[4] = {0, 0, 0, 0};
};

namespace {

void* dalloc(shhd_engine* e, size_t bytes) {
    if (bytes == 0) return nullptr;
    void* p = nullptr;
    const cudaError_t rc = cudaMalloc(&p, bytes);
    if (rc != cudaSuccess) {
        cudaGetLastError();
        throw Failure(SHHD_ENOMEM, "device allocation of " + std::to_string(bytes) + " bytes failed: " + cudaGetErrorString(rc));
    }
    e->device_bytes += bytes;
    return p;
}

void free_engine(shhd_engine* e) {
    for (void* p : {static_cast<void*>(e->k0_u), static_cast<void*>(e->k0_s1), static_cast<void*>(e->k0_s2)})
        if (p) cudaFree(p);
    for (void* p : {e->u, e->s1, e->s2, e->i1, e->i2, e->ext_a, e->ext_b, e->det, e->tw_x, e->tw_y, e->tw_reg, e->phys, e->ref_stage,
                    static_cast<void*>(e->rho0_dev), static_cast<void*>(e->err_dev), static_cast<void*>(e->static_dev),
                    static_cast<void*>(e->members_dev),
                    static_cast<void*>(e->flag_dev), static_cast<void*>(e->ic_scratch), e->meas.tw_x, e->meas.tw_y, e->meas.i1,
                    e->meas.member, static_cast<void*>(e->meas.scratch), static_cast<void*>(e->flux0.acc), static_cast<void*>(e->meas.profile),
                    static_cast<void*>(e->meas.flag), static_cast<void*>(e->meas.line), static_cast<void*>(e->fline[0].acc),
                    static_cast<void*>(e->fline[1].acc), static_cast<void*>(const_cast<double2*>(e->fline[0].wtab)),
                    static_cast<void*>(const_cast<double2*>(e->fline[1].wtab))})
        if (p) cudaFree(p);
    for (auto& kv : e->graphs) cudaGraphExecDestroy(kv.second.exec);
    e->graphs.clear();
    if (e->sk_dev) cudaFree(e->sk_dev);
    if (e->l2_dev) cudaFree(e->l2_dev);
    for (const void* p : {static_cast<const void*>(e->gk.modes), static_cast<const void*>(e->gk.flux_step), static_cast<const void*>(e->gk.integral),
                          static_cast<const void*>(e->gk.sums), static_cast<const void*>(e->gk.wtab)})
        if (p) cudaFree(const_cast<void*>(p));
    if (e->step_dev) cudaFree(e->step_dev);
    for (auto& pe : e->pending) { e->event_pool.push_back(pe.a); e->event_pool.push_back(pe.b); }
    for (cudaEvent_t ev : e->event_pool) cudaEventDestroy(ev);
    if (e->stream) cudaStreamDestroy(e->stream);
}

// --- per-kernel timing (CUDA events around each launch while profiling) ---
cudaEvent_t take_event(shhd_engine* e) {
    if (!e->event_pool.empty()) {
        cudaEvent_t ev = e->event_pool.back();
        e->event_pool.pop_back();
        return ev;
    }
    cudaEvent_t ev;
    check_cuda(cudaEventCreate(&ev), "cudaEventCreate");
    return ev;
}

struct LaunchScope {
    shhd_engine* e;
    int kind;
    cudaEvent_t a = nullptr, b = nullptr;
    LaunchScope(shhd_engine* eng, int k, double bytes) : e(eng), kind(k) {
        e->kernel_launches[kind] += 1;
        e->kernel_bytes[kind] += bytes;
        if (e->profiling) {
            a = take_event(e);
            b = take_event(e);
            check_cuda(cudaEventRecord(a, e->stream), "cudaEventRecord");
        }
    }
    ~LaunchScope() {
        if (a) {
            cudaEventRecord(b, e->stream);
            e->pending.push_back({kind, a, b});
        }
    }
};

void resolve_timings(shhd_engine* e) {
    for (auto& pe : e->pending) {
        float ms = 0.f;
        check_cuda(cudaEventElapsedTime(&ms, pe.a, pe.b), "cudaEventElapsedTime");
        e->kernel_ms[pe.kind] += ms;
        e->event_pool.push_back(pe.a);
        e->event_pool.push_back(pe.b);
    }
    e->pending.clear();
}

void validate_config(const shhd_config& c) {
    if (c.active_nx <= 0 || c.active_ny <= 0) throw Failure(SHHD_EINVAL, "grid sizes must be positive");
    if (c.active_nx % 2 != 0 || c.active_ny % 2 != 0) throw Failure(SHHD_EINVAL, "grid must be even.");
    if (c.nx < c.active_nx || c.ny < c.active_ny) throw Failure(SHHD_EINVAL, "active grid cannot exceed compute grid.");
    if (c.lx <= 0 || c.ly <= 0) throw Failure(SHHD_EINVAL, "domain lengths must be positive");
    if (c.dt <= 0) throw Failure(SHHD_EINVAL, "timestep must be positive");
    if (c.mode < 0 || c.mode > 2) throw Failure(SHHD_EINVAL, "unknown time_evolution mode");
    if (c.integrator < 0 || c.integrator > 1) throw Failure(SHHD_EINVAL, "unknown time_evolution integrator");
    if (c.num_order_parameters < 0 || c.num_order_parameters > SHHD_MAX_ORDER_PARAMETERS)
        throw Failure(SHHD_EUNSUPPORTED, "order_parameters must be in [0, " + std::to_string(SHHD_MAX_ORDER_PARAMETERS) + "]");
    if (c.eta < 0 || c.zeta < 0) throw Failure(SHHD_EINVAL, "transport coefficient requires nonnegative eta and zeta.");
    if (c.cT < 0) throw Failure(SHHD_EINVAL, "thermodynamics requires nonnegative cT.");
    for (int a = 0; a < c.num_order_parameters; ++a) {
        if (c.mobility[a] < 0) throw Failure(SHHD_EINVAL, "transport coefficient requires nonnegative order parameter mobility.");
        if (c.mu_u3[a] < 0) throw Failure(SHHD_EINVAL, "phi4 free energy requires nonnegative u coefficient.");
    }
    if (c.free_energy == SHHD_FE_PLUGIN && (c.fe_plugin < 1 || c.fe_plugin > plugin_count()))
        throw Failure(SHHD_EINVAL, "free-energy plugin style " + std::to_string(c.fe_plugin) + " is not compiled into this library");
    if (c.batch < 1) throw Failure(SHHD_EINVAL, "batch must be >= 1");
    // members are a y or z grid dimension of the stage kernels
    if (c.batch > 65535) throw Failure(SHHD_EINVAL, "batch must be <= 65535");
    if (c.precision != SHHD_FP64 && c.precision != SHHD_FP32) throw Failure(SHHD_EINVAL, "unknown precision");
    if (c.n_sine_forces < 0 || c.n_sine_forces > SHHD_MAX_FORCES || c.n_gradient_forces < 0 || c.n_gradient_forces > SHHD_MAX_FORCES)
        throw Failure(SHHD_EINVAL, "too many forces");
    const bool quiescent = c.mode == SHHD_QUIESCENT;
    if (quiescent && (c.momentum_advection || c.order_parameter_advection))
        throw Failure(SHHD_EINVAL, "quiescent time evolution cannot use nonlinear advection.");
    if (quiescent && c.n_gradient_forces > 0) throw Failure(SHHD_EINVAL, "force/gradient cannot be used in quiescent mode.");
    if (c.ny % 2 == 1 && c.ny > 1) {
        // odd compute rows are handled (the last row pair holds one row)
    }
}

// Row pass of the pair path: outputs are transformed two at a time; pairing
// outputs of one kind (mu_0 with mu_1, psi_0 vx with psi_1 vx, vx with vy, ...)
// keeps the packed product arithmetic uniform.  Each product is written as a
// combination of the terms psi^3, psi vx, psi vy, vx, vy, jx vx, jx vy, jy vy.
void plan_row_pairs(StepPlan& P) {
    std::vector<int> order(P.n_out);
    for (int o = 0; o < P.n_out; ++o) order[o] = o;
    // pairing order: same kinds together, (vx, vy) and (jx vx, jy vy) adjacent
    auto rank = [](int kind) {
        switch (kind) {
            case OUT_MU: return 0;
            case OUT_PSIVX: return 1;
            case OUT_PSIVY: return 2;
            case OUT_VX: return 3;
            case OUT_VY: return 4;
            case OUT_PXX: return 5;
            case OUT_PYY: return 6;
            case OUT_PXY: return 7;
            default: return 8;
        }
    };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return rank(P.out_kind[a]) != rank(P.out_kind[b]) ? rank(P.out_kind[a]) < rank(P.out_kind[b]) : P.out_arg[a] < P.out_arg[b];
    });
    auto coef = [&](int o, float* c) {
        for (int q = 0; q < 8; ++q) c[q] = 0.f;
        const int a = P.out_arg[o];
        switch (P.out_kind[o]) {
            case OUT_MU: c[0] = static_cast<float>(P.mu_u3[a]); break;
            case OUT_PSIVX: c[1] = 1.f; break;
            case OUT_PSIVY: c[2] = 1.f; break;
            case OUT_GRAD: c[3] = static_cast<float>(P.grad_ax[a]); c[4] = static_cast<float>(P.grad_ay[a]); break;
            case OUT_VX: c[3] = 1.f; break;
            case OUT_VY: c[4] = 1.f; break;
            case OUT_PXX: c[5] = 1.f; break;
            case OUT_PXY: c[6] = 1.f; break;
            default: c[7] = 1.f; break;
        }
    };
    P.rp_n = 0;
    for (size_t i = 0; i < order.size(); i += 2) {
        const int pi = P.rp_n++;
        P.rp_a[pi] = order[i];
        P.rp_b[pi] = i + 1 < order.size() ? order[i + 1] : -1;
        float ca[8], cb[8];
        coef(P.rp_a[pi], ca);
        if (P.rp_b[pi] >= 0) coef(P.rp_b[pi], cb);
        else for (int q = 0; q < 8; ++q) cb[q] = 0.f;
        for (int q = 0; q < 8; ++q) { P.rp_coef[pi][q][0] = ca[q]; P.rp_coef[pi][q][1] = cb[q]; }
    }
    // canonical input roles after the x-inverse
    const int s_rho = P.in_slot[0], s_jx = P.in_slot[P.nop + 1], s_jy = P.in_slot[P.nop + 2];
    P.rp_canon = 0; P.rp_prep = 0; P.rp_jline = -1; P.rp_vline = -1;
    if (P.fe_plugin) {
        // plugin styles: mu from every order parameter, per row (row_product_general)
    } else if (!P.need_v) {
        P.rp_canon = 1;
    } else if (P.mode == SHHD_COMPRESSIBLE) {
        if (s_rho >= 0 && s_rho % 2 == 0 && s_jx == s_rho + 1 && s_jy == s_rho + 2 && P.n_in == s_rho + 3) {
            P.rp_canon = 1; P.rp_prep = 1; P.rp_jline = s_rho / 2; P.rp_vline = s_rho / 2 + 1;
        }
    } else if (s_jx >= 0 && s_jx % 2 == 0 && s_jy == s_jx + 1) {
        P.rp_canon = 1; P.rp_jline = s_jx / 2;
    }
    // pairs whose two products are elementwise products of whole input lines
    for (int pi = 0; pi < P.rp_n; ++pi) {
        P.rp_mode[pi] = 0;
        if (!P.rp_canon) continue;
        const int a = P.rp_a[pi], b = P.rp_b[pi];
        const int ka = P.out_kind[a], kb = b >= 0 ? P.out_kind[b] : -1;
        if (ka == OUT_VX && kb == OUT_VY) { P.rp_mode[pi] = 1; continue; }
        if (ka == OUT_PXX && kb == OUT_PYY) { P.rp_mode[pi] = 2; continue; }
        // psi of A in the low half of a line and psi of B (if any) in its high half
        const int sa = P.in_slot[1 + P.out_arg[a]];
        const bool packed = sa >= 0 && sa % 2 == 0 && (b < 0 || (kb == ka && P.in_slot[1 + P.out_arg[b]] == sa + 1));
        if (!packed) continue;
        if (ka == OUT_MU) P.rp_mode[pi] = 3;
        else if (ka == OUT_PSIVX && P.need_v) P.rp_mode[pi] = 4;
        else if (ka == OUT_PSIVY && P.need_v) P.rp_mode[pi] = 5;
    }
    // one input slot and one output (psi -> u psi^3, e.g. quiescent dynamics with N = 1): a
    // pair-line holds two row pairs of that slot instead of a slot and an empty half, both halves
    // with the output's coefficients (blocks of two or more row pairs, i.e. rows of <= 768 points)
    P.rp_pack = 0;
    if (P.n_in == 1 && P.n_out == 1 && P.rp_n == 1 && P.rp_canon && P.rp_mode[0] == 3 && kPairMaxN / P.npx >= 2) {
        P.rp_pack = 1;
        for (int q = 0; q < 8; ++q) P.rp_coef[0][q][1] = P.rp_coef[0][q][0];
    }
}

void build_plan(shhd_engine* e) {
    const shhd_config& c = e->cfg;
    StepPlan& P = e->P;
    std::memset(&P, 0, sizeof(P));
    const int nop = c.num_order_parameters;
    const bool comp = c.mode == SHHD_COMPRESSIBLE, incomp = c.mode == SHHD_INCOMPRESSIBLE, quiet = c.mode == SHHD_QUIESCENT;
    P.nax = c.active_nx; P.nay = c.active_ny;
    P.hx = c.active_nx / 2; P.kyn = c.active_ny - 1;
    P.npx = c.nx; P.npy = c.ny;
    P.kx_unit = 2.0 * M_PI / c.lx;
    P.ky_unit = 2.0 * M_PI / c.ly;
    P.inv_scale = 1.0 / (static_cast<double>(c.nx) * static_cast<double>(c.ny));
    P.nfields = nop + 3; P.nop = nop; P.mode = c.mode; P.batch = c.batch;
    const double grid_size = static_cast<double>(c.nx) * static_cast<double>(c.ny);
    const double volume = c.lx * c.ly;
    const int f_jx = nop + 1, f_jy = nop + 2;

    // ---- physics flags ----
    const bool plugin = c.free_energy == SHHD_FE_PLUGIN;
    const bool has_phys_mu = plugin || (c.free_energy == SHHD_FE_PHI4 && [&] {
        for (int a = 0; a < nop; ++a) if (c.mu_u3[a] != 0.0) return true;
        return false;
    }());
    P.fe_plugin = plugin ? c.fe_plugin : 0;
    for (int k = 0; k < SHHD_MAX_FE_PARAMS; ++k)
        for (int a = 0; a < kMaxOp; ++a) {
            P.fe_param[k][a] = plugin ? c.fe_param[k][a] : 0.0;
            P.fe_paramf[k][a] = static_cast<float>(P.fe_param[k][a]);
        }
    const bool has_visc = c.eta != 0.0 || c.zeta != 0.0;
    P.cT2 = c.cT * c.cT; P.eta = c.eta; P.zeta = c.zeta;
    P.j_zero = quiet || !(P.cT2 != 0.0 || has_visc || c.momentum_advection);
    P.incomp_visc = incomp && c.eta != 0.0 && !P.j_zero;
    for (int a = 0; a < nop; ++a) {
        P.mobility[a] = c.mobility[a];
        P.mu_k0[a] = c.mu_k0[a]; P.mu_k2[a] = c.mu_k2[a]; P.mu_k4[a] = c.mu_k4[a];
        P.mu_u3[a] = (c.free_energy == SHHD_FE_PHI4) ? c.mu_u3[a] : 0.0;
        P.psi_zero[a] = (c.mobility[a] == 0.0 && !c.order_parameter_advection);
        P.psi_linear[a] = c.mobility[a] != 0.0 && (c.mu_k0[a] != 0.0 || c.mu_k2[a] != 0.0 || c.mu_k4[a] != 0.0);
    }
    bool any_grad_incomp = false;
    for (int g = 0; g < c.n_gradient_forces; ++g) {
        const shhd_gradient_force& f = c.gradient_forces[g];
        if (f.component < 0 || f.component >= nop) throw Failure(SHHD_EINVAL, "force/gradient component out of range");
        if (P.psi_zero[f.component]) continue;
        if (f.direction == 0) P.grad_ax[f.component] += -f.amplitude;
        else P.grad_ay[f.component] += -f.amplitude;
        if (incomp) { P.grad_incomp[f.component] = 1; any_grad_incomp = true; }
    }
    // sine sources (fcalculator.cc:702-774)
    for (int s = 0; s < c.n_sine_forces; ++s) {
        const shhd_sine_force& f = c.sine_forces[s];
        int field;
        if (f.target == 0) {
            if (quiet) continue;
            field = f.component == 0 ? f_jx : f_jy;
        } else {
            if (f.component < 0 || f.component >= nop) throw Failure(SHHD_EINVAL, "force/sine component out of range");
            field = 1 + f.component;
        }
        const double im = -0.5 * f.amplitude * grid_size;
        const int gx = f.axis == 0 ? f.nk : 0;
        const int ky = f.axis == 0 ? 0 : f.nk;
        auto add = [&](int gxx, int kyy, double re_, double im_) {
            if (gxx >= P.hx || std::abs(kyy) >= c.active_ny / 2) return;  // only active modes receive the source
            if (P.n_sine >= kMaxSine) throw Failure(SHHD_EUNSUPPORTED, "too many sine sources");
            SineSrc& d = P.sine[P.n_sine++];
            d.field = field; d.gx = gxx; d.ky = kyy; d.re = re_; d.im = im_;
        };
        add(gx, ky, 0.0, im);
        if (f.axis == 1) add(0, -f.nk, 0.0, -im);
    }

    // ---- outputs and groups ----
    auto add_out = [&](int kind, int arg) {
        if (P.n_out >= kMaxOut) throw Failure(SHHD_EUNSUPPORTED, "too many product fields");
        P.out_kind[P.n_out] = kind;
        P.out_arg[P.n_out] = arg;
        return P.n_out++;
    };
    auto add_group_out = [&](int g, int o) {
        if (P.group_nout[g] >= kMaxGroupOut) throw Failure(SHHD_EUNSUPPORTED, "too many products in one group");
        P.group_out[g][P.group_nout[g]++] = o;
    };
    bool need[kMaxFields] = {false};
    bool need_v = false;
    for (int a = 0; a < nop; ++a) {
        const int g = P.n_groups++;
        P.group_kind[g] = GROUP_PSI;
        P.group_alpha[g] = a;
        if (P.psi_zero[a]) continue;
        if (c.mobility[a] != 0.0 && has_phys_mu && (plugin || P.mu_u3[a] != 0.0)) {
            add_group_out(g, add_out(OUT_MU, a));
            need[1 + a] = true;
            if (plugin)  // a plugin's mu_a may read every order parameter
                for (int b = 0; b < nop; ++b) need[1 + b] = true;
        }
        if (c.order_parameter_advection) {
            add_group_out(g, add_out(OUT_PSIVX, a));
            add_group_out(g, add_out(OUT_PSIVY, a));
            need[1 + a] = true;
            need_v = true;
        }
        if (comp && (P.grad_ax[a] != 0.0 || P.grad_ay[a] != 0.0 || [&] {
                for (int q = 0; q < c.n_gradient_forces; ++q) if (c.gradient_forces[q].component == a) return true;
                return false;
            }())) {
            add_group_out(g, add_out(OUT_GRAD, a));
            need_v = true;
        }
    }
    if (!quiet) {
        const int g = P.n_groups++;
        P.group_kind[g] = GROUP_MOMENTUM;
        P.group_alpha[g] = 0;
        if (!P.j_zero) {
            if (comp && has_visc) {
                add_group_out(g, add_out(OUT_VX, 0));
                add_group_out(g, add_out(OUT_VY, 0));
                need_v = true;
            }
            if (c.momentum_advection) {
                add_group_out(g, add_out(OUT_PXX, 0));
                add_group_out(g, add_out(OUT_PXY, 0));
                add_group_out(g, add_out(OUT_PYY, 0));
                need_v = true;
            }
        }
    }
    if (need_v) { need[f_jx] = need[f_jy] = true; if (comp) need[0] = true; }
    P.need_v = need_v ? 1 : 0;
    for (int f = 0; f < kMaxFields; ++f) P.in_slot[f] = -1;
    // slot order follows the reference's pack order: psi..., rho, jx, jy
    for (int a = 0; a < nop; ++a) if (need[1 + a]) { P.in_slot[1 + a] = P.n_in; P.in_field[P.n_in++] = 1 + a; }
    if (need[0]) { P.in_slot[0] = P.n_in; P.in_field[P.n_in++] = 0; }
    if (need[f_jx]) { P.in_slot[f_jx] = P.n_in; P.in_field[P.n_in++] = f_jx; }
    if (need[f_jy]) { P.in_slot[f_jy] = P.n_in; P.in_field[P.n_in++] = f_jy; }

    e->n_evolved = comp ? nop + 3 : (incomp ? nop + 2 : nop);
    e->need_rho0 = incomp && (need_v || P.incomp_visc || any_grad_incomp);

    // ---- noise ----
    const bool noise_psi_on = c.noise_order_parameter && nop > 0;
    const double kbt_psi = c.kBT * c.chi;
    for (int a = 0; a < nop; ++a) {
        P.noise_psi[a] = noise_psi_on && c.mobility[a] != 0.0 && kbt_psi != 0.0;
        const double pref = 2.0 * kbt_psi * grid_size * grid_size / volume;
        P.psi_sig2[a] = 0.5 * pref * c.mobility[a];
    }
    P.noise_j = c.noise_momentum && !quiet && c.kBT != 0.0 && has_visc;
    {
        const double pref = 2.0 * c.kBT * grid_size * grid_size / volume;
        P.j_s = std::sqrt(0.5 * pref);
        P.sqrt_eta = std::sqrt(c.eta);
        P.sqrt_zeta = std::sqrt(c.zeta);
    }
    P.seed = static_cast<uint32_t>(c.noise_seed);
    P.member_offset = static_cast<uint32_t>(c.member_offset);
    P.external_noise = c.noise_source == SHHD_NOISE_EXTERNAL;

    // ---- transforms and launch shapes ----
    P.fy = make_fft_plan(c.ny);
    P.fx = make_fft_plan(c.nx);
    const int cs = static_cast<int>(e->csize);
    const size_t smem_cap = 227 * 1024;
    int W = 1;
    // compile-time kernels: fixed column width per (precision, NY) with one
    // thread group per column; fixed row groups per (precision, NX)
    with_size(c.ny, [&](auto fy) {
        constexpr int FY = decltype(fy)::value;
        if constexpr (FY != 0) {
            const int wf = e->fp32 ? col_width<float, FY>() : col_width<double, FY>();
            const size_t fwd_b = (static_cast<size_t>(wf) * FY + 2ull * wf * P.kyn) * cs;
            if (P.hx % wf == 0 && fwd_b <= smem_cap) {
                e->col_fixed = true;
                W = wf;
                e->smem_col = fwd_b;
                e->smem_col_inv = static_cast<size_t>(wf) * FY * cs;
            }
        }
    });
    with_size(c.nx, [&](auto fx) {
        constexpr int FX = decltype(fx)::value;
        if constexpr (FX != 0) {
            const int gsz = e->fp32 ? row_group<float, FX>() : row_group<double, FX>();
            const bool big = e->fp32 ? row_big_lines<float, FX>() : row_big_lines<double, FX>();
            const size_t rb = static_cast<size_t>(P.n_in + kThreads / gsz) * FX * cs;  // inputs + one work line per group
            const size_t rb2 = static_cast<size_t>(P.n_in + 2) * FX * cs;              // two groups, two work lines
            if (big && rb2 <= smem_cap) {
                e->row_fixed = true;
                e->row_nt = 2 * kThreads;
                e->smem_row = rb2;
            } else if (rb <= smem_cap) {
                e->row_fixed = true;
                e->row_nt = kThreads;
                e->smem_row = rb;
            }
        }
    });
    // shared-memory twiddle tables of the runtime-plan kernels (the compile-time
    // kernels read per-stage rows from global memory)
    P.twy_count = e->col_fixed ? 0 : kTwLo + P.fy.tw_hi_count;
    P.twx_count = e->row_fixed ? 0 : kTwLo + P.fx.tw_hi_count;
    if (!e->col_fixed) {
        // runtime-plan column tile: largest power of two <= 8 dividing Hx whose
        // ping-pong tile pair fits ~100 KB and whose positions fit the register budget
        const size_t col_target = 100 * 1024;
        auto col_bytes = [&](int w) { return static_cast<size_t>(P.twy_count + 2L * w * c.ny) * cs; };
        const long pos_cap = (e->fp32 ? 8L : 4L) * kThreads;
        W = 8;
        while (W > 1 && (P.hx % W != 0 || col_bytes(W) > col_target || static_cast<long>(W) * P.kyn > pos_cap)) W /= 2;
        if (static_cast<long>(W) * P.kyn > 16L * kThreads || col_bytes(W) > smem_cap)
            throw Failure(SHHD_EUNSUPPORTED, "compute grid " + std::to_string(c.ny) + " too large for the column kernels");
        e->smem_col = col_bytes(W);
        e->smem_col_inv = e->smem_col;
        const long posn = static_cast<long>(W) * P.kyn;
        e->npos = posn <= 4L * kThreads ? 4 : (posn <= 8L * kThreads ? 8 : 16);
    }
    P.W = W;
    P.logw = W == 8 ? 3 : (W == 4 ? 2 : (W == 2 ? 1 : 0));
    P.ntiles = P.hx / W;
    P.fy.swz = swizzle_mask(c.ny, e->fp32 ? 16 : 8, W);
    P.fx.swz = swizzle_mask(c.nx, e->fp32 ? 16 : 8, 1);
    if (!e->row_fixed) {
        // runtime-plan row pass: n_in physical lines + lb product lines + lb ping-pong lines
        const size_t line_bytes = static_cast<size_t>(c.nx) * cs;
        const size_t tw_bytes = static_cast<size_t>(P.twx_count) * cs;
        auto row_bytes = [&](int lb) { return tw_bytes + (P.n_in + 2 * lb) * line_bytes; };
        int lb = 4;
        while (lb > 1 && row_bytes(lb) > 113 * 1024) lb /= 2;
        if (row_bytes(lb) > smem_cap) throw Failure(SHHD_EUNSUPPORTED, "row pass does not fit shared memory at this grid and precision");
        P.row_lb = lb;
        P.row_nb = lb;
        e->smem_row = row_bytes(lb);
    }
    P.npos = e->npos;
    P.div_w = make_fastdiv(W);
    P.div_kyn = make_fastdiv(P.kyn);
    P.kyp = (P.kyn + 7) & ~7;
    P.div_kyp = make_fastdiv(P.kyp);
    P.div_npy = make_fastdiv(c.ny);
    P.div_hx = make_fastdiv(P.hx);

    // FP32 pair-line kernels: both compute sizes in 96 ... 1536, column pairs
    // that tile the active kx range, row pairs that tile the compute rows
    if (e->family_override != 0 && e->fp32 && is_pair_size(c.nx) && is_pair_size(c.ny) && P.hx % 2 == 0) {
        const int cp = kPairMaxN / c.ny, rp = kPairMaxN / c.nx;
        const int nip = (P.n_in + 1) / 2;
        const size_t row_b = static_cast<size_t>(rp) * (nip + 1) * c.nx * 16;
        const size_t col_b = static_cast<size_t>(cp) * c.ny * 16 + 3ull * cp * ((P.kyn + 7) & ~7) * 16;  // lines, at most 3 per-mode arrays
        if ((P.hx / 2) % cp == 0 && (c.ny / 2) % rp == 0 && row_b <= smem_cap && col_b <= smem_cap) {
            e->pair_path = true;
            e->col_fixed = e->row_fixed = false;
            W = 2;
            P.W = 2;
            P.logw = 1;
            P.ntiles = P.hx / 2;
            P.div_w = make_fastdiv(2);
            P.twx_count = P.twy_count = 0;
            e->smem_col_inv = static_cast<size_t>(cp) * c.ny * 16;
            e->smem_row = row_b;
            e->smem_col = col_b;
            plan_row_pairs(P);
            // the density as a group of its own (compressible): its update needs no products, and
            // the momentum blocks, the heaviest, lose a field; launch order momentum, order
            // parameters, density (heaviest first, so that the light blocks fill the tail)
            int gm = -1;
            for (int g = 0; g < P.n_groups; ++g)
                if (P.group_kind[g] == GROUP_MOMENTUM) gm = g;
            if (P.mode == SHHD_COMPRESSIBLE && gm >= 0) {
                const int g = P.n_groups++;
                P.group_kind[g] = GROUP_RHO;
                P.group_alpha[g] = 0;
                P.group_nout[g] = 0;
                P.rho_split = 1;
            }
            // per-mode arrays a block uses: acc0 (every group), acc1 (momentum: jy), acc2 (momentum
            // with the density unsplit); shared memory for what this plan's groups use
            const int narr = gm < 0 ? 1 : (P.rho_split ? 2 : 3);
            e->smem_col = static_cast<size_t>(cp) * c.ny * 16 + static_cast<size_t>(narr) * cp * ((P.kyn + 7) & ~7) * 16;
            int k = 0;
            if (gm >= 0) P.group_order[k++] = gm;
            for (int g = 0; g < P.n_groups; ++g)
                if (P.group_kind[g] == GROUP_PSI) P.group_order[k++] = g;
            for (int g = 0; g < P.n_groups; ++g)
                if (P.group_kind[g] == GROUP_RHO) P.group_order[k++] = g;
        }
    }
    // split row pass (every pair-line size)
    e->split_row = e->pair_path && e->family_override == 3 && split_row_supported(c.nx) && c.ny % 2 == 0;
    if (e->split_row) P.rp_pack = 0;  // the split kernels transform unpacked lines
    // row pass over two output pairs at a time (compressible canonical layouts), when selected:
    // level with the pair-line row pass on 1536-point rows (102.5 against 103 us at 1024^2, N = 2;
    // 63 against 56 us with N = 0, where the pair-line kernel runs three blocks per SM), slower on
    // shorter rows, so the default stays the pair-line row pass and the autotuner times both
    e->dual_row = false;
    if (e->pair_path && e->family_override == 4 && c.ny % 2 == 0 && dual_row_supported(P)) {
        e->smem_dual = dual_row_smem_bytes(P);
        e->dual_row = e->smem_dual <= smem_cap;
    }
    // register-resident row pass (1536-point rows of the pair-line layout)
    e->reg_row = false;
    if (e->pair_path && e->family_override == 2 && c.nx == kRegRowN && c.ny % 2 == 0 && P.rp_canon && rrow_rounds(P) >= 2 &&
        rrow_rounds(P) <= 4) {
        e->smem_rrow = rrow_smem_bytes(P);
        e->reg_row = e->smem_rrow <= smem_cap;
    }

    e->state_elems = static_cast<size_t>(P.nfields) * P.hx * P.kyn;
    e->i1_elems = static_cast<size_t>(P.n_in) * P.hx * c.ny;
    e->i2_elems = static_cast<size_t>(P.n_out) * P.hx * c.ny;
}

// kernel dispatch -------------------------------------------------------------
// The dynamic shared-memory limit is a property of the kernel on a device, shared
// by every engine that launches it: only ever raise it, so that an engine with a
// smaller need never lowers the limit below what another engine launches with.
void raise_smem_limit(const void* fn, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<int, const void*>, size_t> limit;
    int dev = 0;
    check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    std::lock_guard<std::mutex> lock(mu);
    size_t& cur = limit[{dev, fn}];
    if (bytes <= cur) return;
    check_cuda(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)), "cudaFuncSetAttribute");
    cur = bytes;
}

template <typename T>
void set_smem_attrs(shhd_engine* e) {
    auto setattr = [](const void* fn, size_t bytes) { raise_smem_limit(fn, bytes); };
    if constexpr (std::is_same<T, float>::value) {
        if (e->pair_path) {
            with_pair_size(e->P.npy, [&](auto fy) {
                constexpr int FY = decltype(fy)::value;
                if constexpr (FY != 0) {
                    setattr(reinterpret_cast<const void*>(pcol_inverse<FY>), e->smem_col_inv);
                    setattr(reinterpret_cast<const void*>(pcol_forward<FY>), e->smem_col);
                    if constexpr (FY >= 384) setattr(reinterpret_cast<const void*>(pcol_forward<FY, 4>), e->smem_col);
                }
            });
            with_pair_size(e->P.npx, [&](auto fx) {
                constexpr int FX = decltype(fx)::value;
                if constexpr (FX != 0) {
                    setattr(reinterpret_cast<const void*>(prow_pass<FX, 2>), e->smem_row);
                    setattr(reinterpret_cast<const void*>(prow_pass<FX, 3>), e->smem_row);
                }
            });
            return;
        }
    }
    with_size(e->P.npy, [&](auto fy) {
        constexpr int FY = decltype(fy)::value;
        if constexpr (FY != 0) {
            if (e->col_fixed) {
                setattr(reinterpret_cast<const void*>(col_inverse_fixed<T, FY>), e->smem_col_inv);
                setattr(reinterpret_cast<const void*>(col_forward_fixed<T, FY>), e->smem_col);
                return;
            }
        }
        setattr(reinterpret_cast<const void*>(col_inverse_kernel<T, 0>), e->smem_col);
        if (e->npos == 4) setattr(reinterpret_cast<const void*>(col_forward_kernel<T, 4, 0>), e->smem_col);
        else if (e->npos == 8) setattr(reinterpret_cast<const void*>(col_forward_kernel<T, 8, 0>), e->smem_col);
        else setattr(reinterpret_cast<const void*>(col_forward_kernel<T, 16, 0>), e->smem_col);
    });
    with_size(e->P.npx, [&](auto fx) {
        constexpr int FX = decltype(fx)::value;
        if constexpr (FX != 0) {
            if (e->row_fixed) {
                if constexpr (row_big_lines<T, FX>()) {
                    if (e->row_nt == 2 * kThreads) {
                        setattr(reinterpret_cast<const void*>(row_pass_fixed<T, FX, 2 * kThreads>), e->smem_row);
                        return;
                    }
                }
                setattr(reinterpret_cast<const void*>(row_pass_fixed<T, FX, kThreads>), e->smem_row);
                return;
            }
        }
        setattr(reinterpret_cast<const void*>(row_pass_kernel<T, 0>), e->smem_row);
    });
}

template <typename T>
void launch_col_inverse(shhd_engine* e, const void* state) {
    const StepPlan& P = e->P;
    if (P.n_in == 0) return;
    dim3 grid(P.ntiles, P.n_in, P.batch);
    const double s = sizeof(cplx<T>);
    LaunchScope scope(e, 0, s * P.batch * P.n_in * (static_cast<double>(P.hx) * P.kyn + static_cast<double>(P.hx) * P.npy));
    auto* st = static_cast<const cplx<T>*>(state);
    auto* i1 = static_cast<cplx<T>*>(e->i1);
    auto* tw = static_cast<const cplx<T>*>(e->tw_y);
    if constexpr (std::is_same<T, float>::value) {
        if (e->pair_path) {
            with_pair_size(P.npy, [&](auto fy) {
                constexpr int FY = decltype(fy)::value;
                if constexpr (FY != 0) {
                    dim3 pg(P.ntiles / (kPairMaxN / FY), P.n_in, P.batch);
                    pcol_inverse<FY><<<pg, kThreads, e->smem_col_inv, e->stream>>>(P, e->members_dev, st, reinterpret_cast<ulonglong2*>(i1),
                                                                                 static_cast<const float2*>(e->tw_y));
                }
            });
            check_cuda(cudaGetLastError(), "col_inverse launch");
            return;
        }
    }
    with_size(P.npy, [&](auto fy) {
        constexpr int FY = decltype(fy)::value;
        if constexpr (FY != 0) {
            if (e->col_fixed) {
                col_inverse_fixed<T, FY><<<grid, kThreads, e->smem_col_inv, e->stream>>>(P, e->members_dev, st, i1, tw);
                return;
            }
        }
        col_inverse_kernel<T, 0><<<grid, kThreads, e->smem_col, e->stream>>>(P, e->members_dev, st, i1, tw);
    });
    check_cuda(cudaGetLastError(), "col_inverse launch");
}

// dynamic shared memory per block up to which three pair-line row-pass blocks share an SM (228 KB,
// less 1 KB reserved per block)
constexpr size_t kRowThreeBlockSmem = 75 * 1024;
// and four column-forward blocks
constexpr size_t kColFourBlockSmem = 56 * 1024;

// launch shapes of the pair-line stage kernels: the variant whose registers are budgeted for
// three row-pass blocks per SM (else two), and for four column-forward blocks (else three), each
// as set (shhd_engine_set_launch_shape, the autotuner) or by rule.  The row rule takes three
// where shared memory holds three (one or two input pair-lines on rows of <= 768 points); the
// column rule four where shared memory holds four, on 1536-point columns and for
// order-parameter-only plans (384 and 768 points with a momentum group run faster at three: 66
// against 69 us and 58 against 62 us)
bool row_three_blocks(const shhd_engine* e) {
    return e->row_blocks ? e->row_blocks == 3 : e->smem_row <= kRowThreeBlockSmem;
}

bool col_four_blocks(const shhd_engine* e) {
    const StepPlan& P = e->P;
    if (P.npy < 384) return false;
    if (e->col_blocks) return e->col_blocks == 4;
    bool momentum = false;
    for (int g = 0; g < P.n_groups; ++g) momentum |= P.group_kind[g] == GROUP_MOMENTUM;
    return e->smem_col <= kColFourBlockSmem && (P.npy == kPairMaxN || !momentum);
}

// the pair-line row pass (not the split, two-pair or register one) is the row kernel
bool pair_line_row(const shhd_engine* e) {
    return e->pair_path && !e->split_row && !e->dual_row && !e->reg_row && e->P.n_out > 0;
}

template <typename T>
void launch_row(shhd_engine* e) {
    const StepPlan& P = e->P;
    if (P.n_out == 0) return;
    dim3 grid((P.npy + 1) / 2, P.batch);
    LaunchScope scope(e, 1, static_cast<double>(sizeof(cplx<T>)) * P.batch * (P.n_in + P.n_out) * static_cast<double>(P.hx) * P.npy);
    if constexpr (std::is_same<T, float>::value) {
        if (e->pair_path && e->split_row && e->phys) {
            launch_split_row(P, P.batch, e->stream, e->members_dev, e->i1, e->phys, e->i2, e->tw_x, e->rho0_dev, e->err_dev);
            check_cuda(cudaGetLastError(), "row_pass launch");
            return;
        }
        if (e->pair_path && e->dual_row) {
            launch_dual_row(P, P.batch, e->stream, e->members_dev, e->i1, e->i2, e->tw_x, e->err_dev);
            check_cuda(cudaGetLastError(), "row_pass launch");
            return;
        }
        if (e->pair_path && e->reg_row && e->tw_reg) {
            launch_rrow_pass(P, P.batch, e->smem_rrow, e->stream, e->members_dev, e->i1, e->i2, e->tw_reg, e->rho0_dev, e->err_dev);
            check_cuda(cudaGetLastError(), "row_pass launch");
            return;
        }
        if (e->pair_path) {
            with_pair_size(P.npx, [&](auto fx) {
                constexpr int FX = decltype(fx)::value;
                if constexpr (FX != 0) {
                    dim3 pg(P.npy / 2 / (kPairMaxN / FX), P.batch);
                    auto kern = row_three_blocks(e) ? prow_pass<FX, 3> : prow_pass<FX, 2>;
                    kern<<<pg, kThreads, e->smem_row, e->stream>>>(P, e->members_dev, static_cast<const ulonglong2*>(e->i1),
                                                                   static_cast<ulonglong2*>(e->i2), static_cast<const float2*>(e->tw_x),
                                                                   e->rho0_dev, e->err_dev);
                }
            });
            check_cuda(cudaGetLastError(), "row_pass launch");
            return;
        }
    }
    with_size(P.npx, [&](auto fx) {
        constexpr int FX = decltype(fx)::value;
        if constexpr (FX != 0) {
            if (e->row_fixed) {
                if constexpr (row_big_lines<T, FX>()) {
                    if (e->row_nt == 2 * kThreads) {
                        row_pass_fixed<T, FX, 2 * kThreads><<<grid, 2 * kThreads, e->smem_row, e->stream>>>(
                            P, e->members_dev, static_cast<const cplx<T>*>(e->i1), static_cast<cplx<T>*>(e->i2),
                            static_cast<const cplx<T>*>(e->tw_x), e->rho0_dev, e->err_dev);
                        return;
                    }
                }
                row_pass_fixed<T, FX, kThreads><<<grid, kThreads, e->smem_row, e->stream>>>(
                    P, e->members_dev, static_cast<const cplx<T>*>(e->i1), static_cast<cplx<T>*>(e->i2), static_cast<const cplx<T>*>(e->tw_x), e->rho0_dev,
                    e->err_dev);
                return;
            }
        }
        row_pass_kernel<T, 0><<<grid, kThreads, e->smem_row, e->stream>>>(
            P, e->members_dev, static_cast<const cplx<T>*>(e->i1), static_cast<cplx<T>*>(e->i2), static_cast<const cplx<T>*>(e->tw_x), e->rho0_dev,
            e->err_dev);
    });
    check_cuda(cudaGetLastError(), "row_pass launch");
}

template <typename T>
void launch_col_forward(shhd_engine* e, const StageArgs<T>& A) {
    const StepPlan& P = e->P;
    if (P.n_groups == 0) return;
    dim3 grid(P.ntiles, P.n_groups, P.batch);
    // algorithmic bytes: I2 tiles read; current (and base) read, next written per evolved field;
    // next stage's I1 written when fused
    LaunchScope scope(e, 2, static_cast<double>(sizeof(cplx<T>)) * P.batch *
                                (P.n_out * static_cast<double>(P.hx) * P.npy +
                                 e->n_evolved * static_cast<double>(P.hx) * P.kyn * (A.det_mode ? 1.0 : (2.0 + (A.wb != 0.0 ? 1.0 : 0.0))) +
                                 (A.fused_inverse ? P.n_in * static_cast<double>(P.hx) * P.npy : 0.0)));
    auto* tw = static_cast<const cplx<T>*>(e->tw_y);
    if constexpr (std::is_same<T, float>::value) {
        if (e->pair_path) {
            with_pair_size(P.npy, [&](auto fy) {
                constexpr int FY = decltype(fy)::value;
                if constexpr (FY != 0) {
                    dim3 pg(P.ntiles / (kPairMaxN / FY), P.n_groups, P.batch);
                    auto kern = pcol_forward<FY>;
                    if constexpr (FY >= 384) {
                        if (col_four_blocks(e)) kern = pcol_forward<FY, 4>;
                    }
                    kern<<<pg, kThreads, e->smem_col, e->stream>>>(P, A, static_cast<const float2*>(e->tw_y));
                }
            });
            check_cuda(cudaGetLastError(), "col_forward launch");
            return;
        }
    }
    with_size(P.npy, [&](auto fy) {
        constexpr int FY = decltype(fy)::value;
        if constexpr (FY != 0) {
            if (e->col_fixed) {
                col_forward_fixed<T, FY><<<grid, kThreads, e->smem_col, e->stream>>>(P, A, tw);
                return;
            }
        }
        if (e->npos == 4) col_forward_kernel<T, 4, 0><<<grid, kThreads, e->smem_col, e->stream>>>(P, A, tw);
        else if (e->npos == 8) col_forward_kernel<T, 8, 0><<<grid, kThreads, e->smem_col, e->stream>>>(P, A, tw);
        else col_forward_kernel<T, 16, 0><<<grid, kThreads, e->smem_col, e->stream>>>(P, A, tw);
    });
    check_cuda(cudaGetLastError(), "col_forward launch");
}

// the run's time, advanced one dt per step as the reference's driver does (project.h:134-136),
// so that printed times match its measures digit for digit
void advance_time(shhd_engine* e, int64_t steps) {
    for (int64_t s = 0; s < steps; ++s) e->time += e->cfg.dt;
}

void upload_members(shhd_engine* e) {
    if (!e->members_dirty) return;
    check_cuda(cudaMemcpyAsync(e->members_dev, e->members.data(), sizeof(MemberInfo) * e->members.size(), cudaMemcpyHostToDevice, e->stream),
               "member info upload");
    check_cuda(cudaStreamSynchronize(e->stream), "member info sync");
    e->members_dirty = false;
}

void ensure_rho0(shhd_engine* e) {
    upload_members(e);
    if (!e->need_rho0) return;
    bool changed = false;
    for (int m = 0; m < e->cfg.batch; ++m) {
        if (e->rho0_cached[m] || !e->members[m].active) continue;
        const double r = e->rho0_candidate[m];
        if (r == 0.0) throw Failure(SHHD_EINVAL, "reference density must be nonzero.");
        e->rho0_value[m] = r;
        e->rho0_cached[m] = 1;
        changed = true;
    }
    if (changed)
        check_cuda(cudaMemcpyAsync(e->rho0_dev, e->rho0_value.data(), sizeof(double) * e->cfg.batch, cudaMemcpyHostToDevice, e->stream),
                   "rho0 upload");
}

template <typename T>
void prepare_static(shhd_engine* e) {
    if (e->n_static == 0) return;
    // about 2048 blocks over all static fields and members (a chunk holds at least one kx = 0 line,
    // so block 0 of a field holds that line)
    const size_t fstride = static_cast<size_t>(e->P.hx) * e->P.kyn;
    const size_t total = fstride * e->n_static * e->P.batch;
    const size_t chunk = std::max<size_t>({static_cast<size_t>(e->P.kyn), (total + 2047) / 2048, static_cast<size_t>(kThreads)});
    dim3 grid(static_cast<unsigned>((fstride + chunk - 1) / chunk), e->n_static, e->P.batch);
    LaunchScope scope(e, 3, static_cast<double>(sizeof(cplx<T>)) * e->P.batch * e->n_static * 3.0 * e->P.hx * e->P.kyn);
    prepare_static_kernel<T><<<grid, kThreads, 0, e->stream>>>(e->P, e->static_dev, static_cast<cplx<T>*>(e->u), static_cast<cplx<T>*>(e->s1),
                                                             static_cast<cplx<T>*>(e->s2), e->k0_u, e->k0_s1, e->k0_s2, static_cast<int>(chunk));
    check_cuda(cudaGetLastError(), "prepare_static launch");
}

constexpr double kSqrt2 = 1.41421356237309504880;
constexpr double kSqrt3 = 1.73205080756887729352;
// time_integrator_srk3_compressible.h:10-21
const double kBeta[3] = {(2.0 * kSqrt2 + kSqrt3) / 5.0, (-4.0 * kSqrt2 + 3.0 * kSqrt3) / 5.0, (kSqrt2 - 2.0 * kSqrt3) / 10.0};
const double kWb[3] = {0.0, 3.0 / 4.0, 1.0 / 3.0};
const double kWc[3] = {1.0, 1.0 / 4.0, 2.0 / 3.0};

template <typename T>
StageArgs<T> stage_args(shhd_engine* e, const void* cur, const void* base, void* next, double wb, double wc, double beta, int srk3, int fused) {
    StageArgs<T> A{};
    A.members = e->members_dev;
    A.cur = static_cast<const cplx<T>*>(cur);
    A.base = static_cast<const cplx<T>*>(base);
    A.next = static_cast<cplx<T>*>(next);
    A.i2 = static_cast<const cplx<T>*>(e->i2);
    A.i1_next = static_cast<cplx<T>*>(e->i1);
    A.ext_a = static_cast<const cplx<T>*>(e->ext_a);
    A.ext_b = static_cast<const cplx<T>*>(e->ext_b);
    A.rho0 = e->rho0_dev;
    A.err = e->err_dev;
    auto k0_of = [&](const void* st) -> double2* {
        if (!e->k0_u) return nullptr;
        if (st == e->u) return e->k0_u;
        if (st == e->s1) return e->k0_s1;
        if (st == e->s2) return e->k0_s2;
        return nullptr;
    };
    A.k0_cur = k0_of(cur);
    A.k0_base = k0_of(base);
    A.k0_next = k0_of(next);
    if (!A.k0_cur || !A.k0_base || !A.k0_next) A.k0_cur = A.k0_base = A.k0_next = nullptr;
    A.wb = wb; A.wc = wc; A.beta = beta;
    A.dt = e->cfg.dt;
    A.sdt = std::sqrt(e->cfg.dt);
    A.step_base = e->step_dev;
    A.step_off = 0;
    A.srk3 = srk3;
    A.fused_inverse = fused;
    A.det_mode = 0;
    return A;
}

template <typename T>
void launch_gk_tap(shhd_engine* e, const void* cur, int step_off, double weight, int first, int last) {
    if (!e->gk_on) return;
    const dim3 g(static_cast<unsigned>(e->gk.nmodes), static_cast<unsigned>(e->P.batch));
    gk_tap_kernel<T><<<g, kThreads, 0, e->stream>>>(e->P, e->gk, e->members_dev, static_cast<const T*>(e->i2), static_cast<const cplx<T>*>(cur),
                                                    e->rho0_dev, e->step_dev, step_off, weight, first, last, e->cfg.dt);
    check_cuda(cudaGetLastError(), "gk_tap launch");
}

template <typename T>
void launch_flux0_tap(shhd_engine* e, const void* cur, int step_off, double weight, int first) {
    if (!e->flux0_on) return;
    const double2* k0 = nullptr;
    if (e->k0_u) k0 = cur == e->u ? e->k0_u : (cur == e->s1 ? e->k0_s1 : (cur == e->s2 ? e->k0_s2 : nullptr));
    const dim3 g(static_cast<unsigned>(e->flux0.ncol), static_cast<unsigned>(e->P.batch));
    flux0_tap_kernel<T><<<g, kThreads, 0, e->stream>>>(e->P, e->flux0, e->members_dev, static_cast<const T*>(e->i2),
                                                       static_cast<const cplx<T>*>(cur), k0, weight, first, e->step_dev, step_off);
    check_cuda(cudaGetLastError(), "flux0_tap launch");
}

template <typename T>
void launch_flux_line_taps(shhd_engine* e, const void* cur, int step_off, double weight, int first, int last) {
    for (int ax = 0; ax < 2; ++ax) {
        if (!e->fline_on[ax]) continue;
        const FluxLineArgs& L = e->fline[ax];
        const double2* k0 = nullptr;
        if (e->k0_u) k0 = cur == e->u ? e->k0_u : (cur == e->s1 ? e->k0_s1 : (cur == e->s2 ? e->k0_s2 : nullptr));
        const dim3 g(static_cast<unsigned>((L.nline + kThreads / 32 - 1) / (kThreads / 32)), static_cast<unsigned>(e->P.batch));
        const size_t smem = ax == 1 ? sizeof(double2) * e->P.npy : 0;
        flux_line_tap_kernel<T><<<g, kThreads, smem, e->stream>>>(e->P, L, e->members_dev, static_cast<const T*>(e->i2),
                                                                   static_cast<const cplx<T>*>(cur), k0, e->rho0_dev, e->step_dev, step_off, weight,
                                                                   first, last, e->cfg.dt);
        check_cuda(cudaGetLastError(), "flux_line_tap launch");
    }
}

// the launches of one call of nsteps steps (step indices relative to *step_dev)
template <typename T>
void record_steps(shhd_engine* e, int nsteps) {
    prepare_static<T>(e);
    launch_col_inverse<T>(e, e->u);
    const bool srk3 = e->cfg.integrator == SHHD_SRK3;
    for (int s = 0; s < nsteps; ++s) {
        const bool last_step = (s + 1 == nsteps);
        if (srk3) {
            void* cur[3] = {e->u, e->s1, e->s2};
            void* nxt[3] = {e->s1, e->s2, e->u};
            for (int k = 0; k < 3; ++k) {
                launch_row<T>(e);
                const int fused = !(last_step && k == 2);
                StageArgs<T> A = stage_args<T>(e, cur[k], e->u, nxt[k], kWb[k], kWc[k], kBeta[k], 1, fused);
                A.step_off = s;
                launch_col_forward<T>(e, A);
                // stage flux weights 1/6, 1/6, 2/3 (time_integrator_srk3_compressible.h:15-21)
                launch_gk_tap<T>(e, cur[k], s, k == 2 ? 2.0 / 3.0 : 1.0 / 6.0, k == 0, k == 2);
                launch_flux0_tap<T>(e, cur[k], s, k == 2 ? 2.0 / 3.0 : 1.0 / 6.0, k == 0);
                launch_flux_line_taps<T>(e, cur[k], s, k == 2 ? 2.0 / 3.0 : 1.0 / 6.0, k == 0, k == 2);
            }
        } else {
            launch_row<T>(e);
            StageArgs<T> A = stage_args<T>(e, e->u, e->u, e->s1, 0.0, 1.0, 0.0, 0, last_step ? 0 : 1);
            A.step_off = s;
            launch_col_forward<T>(e, A);
            launch_gk_tap<T>(e, e->u, s, 1.0, 1, 1);
            launch_flux0_tap<T>(e, e->u, s, 1.0, 1);
            launch_flux_line_taps<T>(e, e->u, s, 1.0, 1, 1);
            std::swap(e->u, e->s1);
            std::swap(e->k0_u, e->k0_s1);
        }
    }
}

void set_step_dev(shhd_engine* e) {
    set_step_kernel<<<1, 1, 0, e->stream>>>(e->step_dev, static_cast<unsigned long long>(e->step_index));
    check_cuda(cudaGetLastError(), "set_step launch");
}

void drop_graphs(shhd_engine* e) {
    for (auto& kv : e->graphs) check_cuda(cudaGraphExecDestroy(kv.second.exec), "cudaGraphExecDestroy");
    e->graphs.clear();
}

// graph sizes a call is split into: the chunk, then every power of two below it
// (even sizes only for Euler, whose two state buffers swap every step)
std::vector<int> graph_sizes(const shhd_engine* e) {
    std::vector<int> s{e->graph_chunk};
    for (int p = 1 << 30; p >= 1; p >>= 1)
        if (p < e->graph_chunk && (e->cfg.integrator != SHHD_EULER || p % 2 == 0)) s.push_back(p);
    return s;
}

// capture one call of K steps (plus the advance of the step counter) as a graph
template <typename T>
shhd_engine::CachedGraph& capture_graph(shhd_engine* e, int K) {
    int64_t l0[4];
    double b0[4];
    for (int k = 0; k < 4; ++k) { l0[k] = e->kernel_launches[k]; b0[k] = e->kernel_bytes[k]; }
    check_cuda(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
    cudaGraph_t g = nullptr;
    try {
        record_steps<T>(e, K);
        advance_step_kernel<<<1, 1, 0, e->stream>>>(e->step_dev, static_cast<unsigned long long>(K));
        check_cuda(cudaGetLastError(), "advance_step launch");
    } catch (...) {
        cudaStreamEndCapture(e->stream, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    check_cuda(cudaStreamEndCapture(e->stream, &g), "cudaStreamEndCapture");
    shhd_engine::CachedGraph cg;
    const cudaError_t rc = cudaGraphInstantiate(&cg.exec, g, 0);
    cudaGraphDestroy(g);
    check_cuda(rc, "cudaGraphInstantiate");
    for (int k = 0; k < 4; ++k) {
        cg.launches[k] = e->kernel_launches[k] - l0[k];
        cg.bytes[k] = e->kernel_bytes[k] - b0[k];
        e->kernel_launches[k] = l0[k];
        e->kernel_bytes[k] = b0[k];
    }
    return e->graphs[K] = cg;
}

template <typename T>
void enqueue_steps(shhd_engine* e, int nsteps) {
    ensure_rho0(e);
    set_step_dev(e);
    int done = 0;
    if (e->graph_chunk > 0 && !e->profiling) {
        for (const int size : graph_sizes(e)) {
            while (nsteps - done >= size) {
                auto it = e->graphs.find(size);
                shhd_engine::CachedGraph& cg = it != e->graphs.end() ? it->second : capture_graph<T>(e, size);
                check_cuda(cudaGraphLaunch(cg.exec, e->stream), "cudaGraphLaunch");
                for (int k = 0; k < 4; ++k) { e->kernel_launches[k] += cg.launches[k]; e->kernel_bytes[k] += cg.bytes[k]; }
                done += size;
            }
        }
        e->step_index += done;
        advance_time(e, done);
        if (done < nsteps) set_step_dev(e);
    }
    if (done < nsteps) {
        record_steps<T>(e, nsteps - done);
        e->step_index += nsteps - done;
        advance_time(e, nsteps - done);
    }
}

void enqueue(shhd_engine* e, int nsteps) {
    if (nsteps < 0) throw Failure(SHHD_EINVAL, "nsteps must be nonnegative");
    if (nsteps == 0) return;
    if (e->cfg.noise_source == SHHD_NOISE_EXTERNAL && nsteps != 1)
        throw Failure(SHHD_EINVAL, "external noise supplies one step at a time: call step with nsteps = 1");
    check_cuda(cudaSetDevice(e->device), "cudaSetDevice");
    if (e->fp32) enqueue_steps<float>(e, nsteps);
    else enqueue_steps<double>(e, nsteps);
}

void sync_and_check(shhd_engine* e) {
    check_cuda(cudaStreamSynchronize(e->stream), "stream synchronize");
    resolve_timings(e);
    int err = 0;
    check_cuda(cudaMemcpy(&err, e->err_dev, sizeof(int), cudaMemcpyDeviceToHost), "error flag read");
    if (err != 0) {
        check_cuda(cudaMemset(e->err_dev, 0, sizeof(int)), "error flag reset");
        if (err & ERR_ZERO_DENSITY) throw Failure(SHHD_ENUMERIC, "compressible velocity encountered zero density.");
        if (err & ERR_NONFINITE)
            throw Failure(SHHD_ENUMERIC, "state is not finite (NaN or Inf) after a step: the integration diverged "
                                         "(timestep outside the stability interval of the stiffest mode, or a state too far from the model's range).");
    }
}

// reference layout <-> active layout (host side) -----------------------------
size_t ref_doubles(const shhd_engine* e) {
    return static_cast<size_t>(e->P.nfields) * (e->cfg.nx / 2 + 1) * e->cfg.ny * 2;
}

// host array (reference layout) -> device staging buffer -> engine layout; the
// inactive-mode check runs on the device over the staged copy
template <typename T>
void upload_ref(shhd_engine* e, const double* ref, void* dst_base, int member, bool check_inactive) {
    const StepPlan& P = e->P;
    const int ref_hx = e->cfg.nx / 2 + 1;
    const size_t bytes = ref_doubles(e) * sizeof(double);
    if (!e->ref_stage) e->ref_stage = dalloc(e, bytes);
    if (!e->flag_dev) e->flag_dev = static_cast<int*>(dalloc(e, sizeof(int)));
    check_cuda(cudaMemcpyAsync(e->ref_stage, ref, bytes, cudaMemcpyHostToDevice, e->stream), "state upload");
    const double2* st = static_cast<const double2*>(e->ref_stage);
    if (check_inactive) {
        check_cuda(cudaMemsetAsync(e->flag_dev, 0, sizeof(int), e->stream), "flag clear");
        dim3 g((P.npy * ref_hx + kThreads - 1) / kThreads, P.nfields);
        check_inactive_kernel<<<g, kThreads, 0, e->stream>>>(P, ref_hx, st, e->flag_dev);
        check_cuda(cudaGetLastError(), "check_inactive launch");
        int bad = 0;
        check_cuda(cudaMemcpyAsync(&bad, e->flag_dev, sizeof(int), cudaMemcpyDeviceToHost, e->stream), "flag read");
        check_cuda(cudaStreamSynchronize(e->stream), "upload sync");
        if (bad) throw Failure(SHHD_EINVAL, "state has a nonzero entry outside the active modes");
    }
    cplx<T>* dst = static_cast<cplx<T>*>(dst_base) + static_cast<size_t>(member) * e->state_elems;
    dim3 g((P.hx * P.kyn + kThreads - 1) / kThreads, P.nfields);
    ref_to_active_kernel<T><<<g, kThreads, 0, e->stream>>>(P, ref_hx, st, dst);
    check_cuda(cudaGetLastError(), "ref_to_active launch");
    check_cuda(cudaStreamSynchronize(e->stream), "state upload sync");
}

template <typename T>
void download_ref(shhd_engine* e, const void* src_base, int member, double* ref) {
    const StepPlan& P = e->P;
    const int ref_hx = e->cfg.nx / 2 + 1;
    const size_t bytes = ref_doubles(e) * sizeof(double);
    if (!e->ref_stage) e->ref_stage = dalloc(e, bytes);
    const cplx<T>* src = static_cast<const cplx<T>*>(src_base) + static_cast<size_t>(member) * e->state_elems;
    dim3 g((P.npy * ref_hx + kThreads - 1) / kThreads, P.nfields);
    active_to_ref_kernel<T><<<g, kThreads, 0, e->stream>>>(P, ref_hx, src, static_cast<double2*>(e->ref_stage));
    check_cuda(cudaGetLastError(), "active_to_ref launch");
    check_cuda(cudaMemcpyAsync(ref, e->ref_stage, bytes, cudaMemcpyDeviceToHost, e->stream), "state download");
    check_cuda(cudaStreamSynchronize(e->stream), "state download sync");
}

template <typename T>
void run_rhs(shhd_engine* e, int member, double* out) {
    const size_t bytes = e->state_elems * e->cfg.batch * sizeof(cplx<T>);
    if (!e->det) e->det = dalloc(e, bytes);
    ensure_rho0(e);
    check_cuda(cudaMemsetAsync(e->det, 0, bytes, e->stream), "det clear");
    launch_col_inverse<T>(e, e->u);
    launch_row<T>(e);
    StageArgs<T> A = stage_args<T>(e, e->u, e->u, e->det, 0.0, 1.0, 0.0, 0, 0);
    A.det_mode = 1;
    launch_col_forward<T>(e, A);
    sync_and_check(e);
    download_ref<T>(e, e->det, member, out);
}

// host twiddle tables of the engine's transforms (bytes), in the format its kernels read
template <typename T>
std::vector<unsigned char> host_twiddles(const shhd_engine* e, int n, bool fixed) {
    std::vector<unsigned char> out;
    if (e->pair_path) {
        with_pair_size(n, [&](auto fn) {
            constexpr int FN = decltype(fn)::value;
            if constexpr (FN != 0) {
                const int cnt = std::max(PairPlan<FN>::c.twsz, 1);
                std::vector<float> t(2 * static_cast<size_t>(cnt), 0.f);
                pair_twiddles_host<FN>(t.data());
                out.resize(t.size() * sizeof(float));
                std::memcpy(out.data(), t.data(), out.size());
            }
        });
        if (out.empty()) throw Failure(SHHD_EUNSUPPORTED, "no pair-path twiddles for size " + std::to_string(n));
        return out;
    }
    const auto t = fixed ? stage_table<T>(n) : twiddle_table<T>(n);
    out.resize(t.size() * sizeof(cplx<T>));
    std::memcpy(out.data(), t.data(), out.size());
    return out;
}

template <typename T>
void init_device(shhd_engine* e) {
    const size_t cs = sizeof(cplx<T>);
    const size_t B = e->cfg.batch;
    e->u = dalloc(e, e->state_elems * B * cs);
    e->s1 = dalloc(e, e->state_elems * B * cs);
    e->s2 = dalloc(e, e->state_elems * B * cs);
    check_cuda(cudaMemsetAsync(e->u, 0, e->state_elems * B * cs, e->stream), "memset");
    check_cuda(cudaMemsetAsync(e->s1, 0, e->state_elems * B * cs, e->stream), "memset");
    check_cuda(cudaMemsetAsync(e->s2, 0, e->state_elems * B * cs, e->stream), "memset");
    e->i1 = dalloc(e, std::max<size_t>(1, e->i1_elems) * B * cs);
    e->i2 = dalloc(e, std::max<size_t>(1, e->i2_elems) * B * cs);
    if (e->cfg.noise_source == SHHD_NOISE_EXTERNAL) {
        e->ext_a = dalloc(e, e->state_elems * B * cs);
        e->ext_b = dalloc(e, e->state_elems * B * cs);
        check_cuda(cudaMemsetAsync(e->ext_a, 0, e->state_elems * B * cs, e->stream), "memset");
        check_cuda(cudaMemsetAsync(e->ext_b, 0, e->state_elems * B * cs, e->stream), "memset");
    }
    const auto twx = host_twiddles<T>(e, e->cfg.nx, e->row_fixed);
    const auto twy = host_twiddles<T>(e, e->cfg.ny, e->col_fixed);
    e->tw_x = dalloc(e, twx.size());
    e->tw_y = dalloc(e, twy.size());
    e->tw_bytes = twx.size() + twy.size();
    check_cuda(cudaMemcpyAsync(e->tw_x, twx.data(), twx.size(), cudaMemcpyHostToDevice, e->stream), "twiddle upload");
    check_cuda(cudaMemcpyAsync(e->tw_y, twy.data(), twy.size(), cudaMemcpyHostToDevice, e->stream), "twiddle upload");
    if (e->fp32 && e->cfg.nx == kRegRowN) {
        std::vector<float> t(reg_twiddle_floats());
        reg_twiddles(t.data());
        e->tw_reg = dalloc(e, t.size() * sizeof(float));
        check_cuda(cudaMemcpyAsync(e->tw_reg, t.data(), t.size() * sizeof(float), cudaMemcpyHostToDevice, e->stream), "twiddle upload");
        check_cuda(cudaStreamSynchronize(e->stream), "twiddle upload");
    }
    e->rho0_dev = static_cast<double*>(dalloc(e, sizeof(double) * B));
    check_cuda(cudaMemsetAsync(e->rho0_dev, 0, sizeof(double) * B, e->stream), "memset");
    e->err_dev = static_cast<int*>(dalloc(e, sizeof(int)));
    e->step_dev = static_cast<unsigned long long*>(dalloc(e, sizeof(unsigned long long)));
    if (e->fp32) {
        const size_t k0b = sizeof(double2) * B * e->P.nfields;
        e->k0_u = static_cast<double2*>(dalloc(e, k0b));
        e->k0_s1 = static_cast<double2*>(dalloc(e, k0b));
        e->k0_s2 = static_cast<double2*>(dalloc(e, k0b));
        for (double2* p : {e->k0_u, e->k0_s1, e->k0_s2}) check_cuda(cudaMemsetAsync(p, 0, k0b, e->stream), "memset");
    }
    e->members_dev = static_cast<MemberInfo*>(dalloc(e, sizeof(MemberInfo) * B));
    e->members.resize(B);
    for (size_t m = 0; m < B; ++m) {
        e->members[m].key = static_cast<uint32_t>(e->cfg.member_offset + static_cast<int>(m));
        e->members[m].active = 1;
        e->members[m].step0 = 0;
        e->members[m].noise_scale = 1.0;
    }
    e->members_dirty = true;
    check_cuda(cudaMemsetAsync(e->err_dev, 0, sizeof(int), e->stream), "memset");
    // fields the integrator does not evolve
    std::vector<int> st;
    const int nop = e->cfg.num_order_parameters;
    if (e->cfg.mode == SHHD_INCOMPRESSIBLE) st = {0};
    if (e->cfg.mode == SHHD_QUIESCENT) st = {0, nop + 1, nop + 2};
    e->n_static = static_cast<int>(st.size());
    if (!st.empty()) {
        e->static_dev = static_cast<int*>(dalloc(e, sizeof(int) * st.size()));
        check_cuda(cudaMemcpyAsync(e->static_dev, st.data(), sizeof(int) * st.size(), cudaMemcpyHostToDevice, e->stream), "static fields upload");
    }
    set_smem_attrs<T>(e);
    check_cuda(cudaStreamSynchronize(e->stream), "init sync");
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

const char* shhd_last_error(void) { return g_last_error.c_str(); }

int shhd_free_energy_plugin_count(void) { return plugin_count(); }

const char* shhd_free_energy_plugin_name(int id) {
    PluginInfo info{};
    return plugin_info(id, &info) ? info.name : nullptr;
}

const char* shhd_free_energy_plugin_key(int id, int k) {
    PluginInfo info{};
    return plugin_info(id, &info) && k >= 0 && k < info.n_params ? info.keys[k] : nullptr;
}

int shhd_engine_create(const shhd_config* cfg, shhd_engine** out) {
    if (!cfg || !out) {
        g_last_error = "null argument";
        return SHHD_EINVAL;
    }
    *out = nullptr;
    shhd_engine* e = new shhd_engine();
    const int rc = guarded([&] {
        e->cfg = *cfg;
        validate_config(e->cfg);
        e->fp32 = cfg->precision == SHHD_FP32;
        e->csize = e->fp32 ? sizeof(float2) : sizeof(double2);
        build_plan(e);
        check_cuda(cudaGetDevice(&e->device), "cudaGetDevice");
        check_cuda(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking), "cudaStreamCreate");
        e->rho0_candidate.assign(cfg->batch, 0.0);
        e->rho0_cached.assign(cfg->batch, 0);
        e->rho0_value.assign(cfg->batch, 0.0);
        if (e->fp32) init_device<float>(e);
        else init_device<double>(e);
    });
    if (rc != SHHD_OK) {
        free_engine(e);
        delete e;
        return rc;
    }
    *out = e;
    return SHHD_OK;
}

void shhd_engine_destroy(shhd_engine* e) {
    if (!e) return;
    cudaSetDevice(e->device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    free_engine(e);
    delete e;
}

int shhd_engine_info(const shhd_engine* e, shhd_info* info) {
    if (!e || !info) { g_last_error = "null argument"; return SHHD_EINVAL; }
    const StepPlan& P = e->P;
    std::memset(info, 0, sizeof(*info));
    info->nfields = P.nfields;
    info->state_doubles = ref_doubles(e);
    info->active_modes = static_cast<size_t>(P.hx) * P.kyn;
    info->n_inverse = P.n_in;
    info->n_forward = P.n_out;
    info->n_evolved = e->n_evolved;
    info->device_bytes = e->device_bytes;
    const double s = static_cast<double>(e->csize);
    const double I = static_cast<double>(P.hx) * P.npy;
    const double Ma = static_cast<double>(P.hx) * P.kyn;
    const double nev = e->n_evolved;
    // steady-state fused stage: row reads F_in*I, writes F_out*I; column forward reads F_out*I,
    // current (and base on stages 2, 3 of SRK3), writes the evolved fields and F_in*I
    const double base_reads = e->cfg.integrator == SHHD_SRK3 ? nev * 2.0 / 3.0 : 0.0;
    info->bytes_per_stage = s * P.batch * (2.0 * P.n_in * I + 2.0 * P.n_out * I + (nev + base_reads + nev) * Ma);
    auto flops = [](double n) { return 5.0 * n * std::log2(n); };
    info->fft_flops_per_stage = P.batch * ((P.n_in + P.n_out) * (P.hx * flops(P.npy) + 0.5 * P.npy * flops(P.npx)));
    info->step_index = e->step_index;
    info->time = e->time;
    return SHHD_OK;
}

int shhd_engine_set_state(shhd_engine* e, int member, const double* state, size_t n) {
    return guarded([&] {
        if (!e || !state) throw Failure(SHHD_EINVAL, "null argument");
        if (member < 0 || member >= e->cfg.batch) throw Failure(SHHD_EINVAL, "member index out of range");
        if (n != ref_doubles(e)) throw Failure(SHHD_EINVAL, "state size mismatch: expected " + std::to_string(ref_doubles(e)) + " doubles");
        check_cuda(cudaSetDevice(e->device), "cudaSetDevice");
        if (e->fp32) upload_ref<float>(e, state, e->u, member, true);
        else upload_ref<double>(e, state, e->u, member, true);
        e->rho0_candidate[member] = state[0] / (static_cast<double>(e->cfg.nx) * e->cfg.ny);
        if (e->k0_u) {  // FP64 copies of the k = 0 modes
            const size_t block = static_cast<size_t>(e->cfg.nx / 2 + 1) * e->cfg.ny * 2;  // doubles per field
            std::vector<double2> k0(e->P.nfields);
            for (int f = 0; f < e->P.nfields; ++f) k0[f] = make_double2(state[f * block], state[f * block + 1]);
            check_cuda(cudaMemcpyAsync(e->k0_u + static_cast<size_t>(member) * e->P.nfields, k0.data(), sizeof(double2) * k0.size(),
                                       cudaMemcpyHostToDevice, e->stream),
                       "k0 upload");
            check_cuda(cudaStreamSynchronize(e->stream), "k0 upload sync");
        }
    });
}

int shhd_engine_get_state(shhd_engine* e, int member, double* state, size_t n) {
    return guarded([&] {
        if (!e || !state) throw Failure(SHHD_EINVAL, "null argument");
        if (member < 0 || member >= e->cfg.batch) throw Failure(SHHD_EINVAL, "member index out of range");
        if (n != ref_doubles(e)) throw Failure(SHHD_EINVAL, "state size mismatch");
        check_cuda(cudaSetDevice(e->device), "cudaSetDevice");
        if (e->fp32) download_ref<float>(e, e->u, member, state);
        else download_ref<double>(e, e->u, member, state);
        if (e->k0_u) {  // the evolved fields' k = 0 modes from their FP64 copies
            std::vector<double2> k0(e->P.nfields);
            check_cuda(cudaMemcpyAsync(k0.data(), e->k0_u + static_cast<size_t>(member) * e->P.nfields, sizeof(double2) * k0.size(),
                                       cudaMemcpyDeviceToHost, e->stream),
                       "k0 download");
            check_cuda(cudaStreamSynchronize(e->stream), "k0 download sync");
            const size_t block = static_cast<size_t>(e->cfg.nx / 2 + 1) * e->cfg.ny * 2;
            const int nop = e->cfg.num_order_parameters;
            for (int f = 0; f < e->P.nfields; ++f) {
                const bool evolved = e->cfg.mode == SHHD_COMPRESSIBLE || (f >= 1 && f <= nop) ||
                                     (e->cfg.mode == SHHD_INCOMPRESSIBLE && f > nop);
                if (!evolved) continue;
                state[f * block] = k0[f].x;
                state[f * block + 1] = k0[f].y;
            }
        }
    });
}

int shhd_engine_set_external_noise(shhd_engine* e, int member, const double* sto_a, const double* sto_b, size_t n) {
    return guarded([&] {
        if (!e || !sto_a) throw Failure(SHHD_EINVAL, "null argument");
        if (e->cfg.noise_source != SHHD_NOISE_EXTERNAL) throw Failure(SHHD_EINVAL, "engine was created with Philox noise");
        if (member < 0 || member >= e->cfg.batch) throw Failure(SHHD_EINVAL, "member index out of range");
        if (n != ref_doubles(e)) throw Failure(SHHD_EINVAL, "noise size mismatch");
        if (e->cfg.integrator == SHHD_SRK3 && !sto_b) throw Failure(SHHD_EINVAL, "srk3 needs both noise draws");
        check_cuda(cudaSetDevice(e->device), "cudaSetDevice");
        if (e->fp32) {
            upload_ref<float>(e, sto_a, e->ext_a, member, false);
            if (sto_b) upload_ref<float>(e, sto_b, e->ext_b, member, false);
        } else {
            upload_ref<double>(e, sto_a, e->ext_a, member, false);
            if (sto_b) upload_ref<double>(e, sto_b, e->ext_b, member, false);
        }
    });
}

int shhd_engine_step(shhd_engine* e, int nsteps) {
    return guarded([&] {
        if (!e) throw Failure(SHHD_EINVAL, "null engine");
        enqueue(e, nsteps);
        sync_and_check(e);
    });
}

int shhd_engine_step_async(shhd_engine* e, int nsteps) {
    return guarded([&] {
        if (!e) throw Failure(SHHD_EINVAL, "null engine");
        enqueue(e, nsteps);
    });
}

int shhd_engine_synchronize(shhd_engine* e) {
    return guarded([&] {
        if (!e) throw Failure(SHHD_EINVAL, "null engine");
        check_cuda(cudaSetDevice(e->device), "cudaSetDevice");
        sync_and_check(e);
    });
}

int shhd_engine_rhs(shhd_engine* e, int member, double* det, size_t n) {
    return guarded([&] {
        if (!e || !det) throw Failure(SHHD_EINVAL, "null argument");
        if (member < 0 || member >= e->cfg.batch) throw Failure(SHHD_EINVAL, "member index out of range");
        if (n != ref_doubles(e)) throw Failure(SHHD_EINVAL, "size mismatch");
        check_cuda(cudaSetDevice(e->device), "cudaSetDevice");
        if (e->fp32) run_rhs<float>(e, member, det);
        else run_rhs<double>(e, member, det);
    });
}

int shhd_engine_set_member(shhd_engine* e, int member, uint32_t key, int64_t step_origin, double noise_scale, int active) {
    return guarded([&] {
        if (!e) throw Failure(SHHD_EINVAL, "null engine");
        if (member < 0 || member >= e->cfg.batch) throw Failure(SHHD_EINVAL, "member index out of range");
        if (!(noise_scale >= 0.0)) throw Failure(SHHD_EINVAL, "noise_scale must be nonnegative");
        MemberInfo& mi = e->members[member];
        mi.key = key;
        mi.step0 = step_origin;
        mi.noise_scale = noise_scale;
        mi.active = active ? 1 : 0;
        e->rho0_cached[member] = 0;  // a new trajectory: rho0 is taken again at its first use
        e->members_dirty = true;
    });
}

int shhd_engine_sk_accumulate(shhd_engine* e, int field) {
    return guarded([&] {
        if (!e) throw Failure(SHHD_EINVAL, "null engine");
        if (field < 0 || field >= e->P.nfields) throw Failure(SHHD_EINVAL, "field index out of range");
        if (e->sk_count > 0 && field != e->sk_field) throw Failure(SHHD_EINVAL, "the accumulator holds another field: read it with reset first");
        check_cuda(cudaSetDevice(e->device), "cudaSetDevice");
        const StepPlan& P = e->P;
        const size_t modes = static_cast<size_t>(P.hx) * P.kyn;
        if (!e->sk_dev) {
            e->sk_dev = static_cast<double*>(dalloc(e, modes * sizeof(double)));
            check_cuda(cudaMemsetAsync(e->sk_dev, 0, modes * sizeof(double), e->stream), "memset");
        }
        int active = 0;
        for (const MemberInfo& m : e->members) active += m.active ? 1 : 0;
        if (active == 0) throw Failure(SHHD_EINVAL, "no active member");
        upload_members(e);
        const double np2 = static_cast<double>(e->cfg.nx) * e->cfg.ny;
        const double scale = e->cfg.lx * e->cfg.ly / (np2 * np2) / active;
        const dim3 g(static_cast<unsigned>((modes + kThreads - 1) / kThreads));
        if (e->fp32)
            structure_factor_kernel<float><<<g, kThreads, 0, e->stream>>>(P, e->members_dev, static_cast<const float2*>(e->u), field, scale, e->sk_dev);
        else
            structure_factor_kernel<double><<<g, kThreads, 0, e->stream>>>(P, e->members_dev, static_cast<const double2*>(e->u), field, scale, e->sk_dev);
        check_cuda(cudaGetLastError(), "structure_factor launch");
        e->sk_field = field;
        e->sk_count += 1;
    });
}

int shhd_engine_sk_read(shhd_engine* e, double* out, size_t n_modes, int64_t* count, int reset) {
    return guarded([&] {
        if (!e || !out) throw Failure(SHHD_EINVAL, "null argument");
        const size_t modes = static_cast<size_t>(e->P.hx) * e->P.kyn;
        if (n_modes != modes) throw Failure(SHHD_EINVAL, "mode count mismatch: expected " + std::to_string(modes));
        check_cuda(cudaSetDevice(e->device), "cudaSetDevice");
        if (count) *count = e->sk_count;
        if (!e->sk_dev || e->sk_count == 0) {
            std::memset(out, 0, modes * sizeof(double));
            return;
        }
        check_cuda(cudaMemcpyAsync(out, e->sk_dev, modes * sizeof(double), cudaMemcpyDeviceToHost, e->stream), "sk download");
        if (reset) check_cuda(cudaMemsetAsync(e->sk_dev, 0, modes * sizeof(double), e->stream), "sk reset");
        check_cuda(cudaStreamSynchronize(e->stream), "sk sync");
        if (reset) { e->sk_count = 0; e->sk_field = -1; }
    });
}

}  // extern "C"

// ---------------------------------------------------------------------------
// autotuner: kernel family x graph chunk, timed on the engine's own state
// ---------------------------------------------------------------------------
namespace {

// switch kernel family: new plan, twiddle tables and shared-memory limits (buffer sizes are
// the same for every family); any captured graph is dropped
template <typename T>
void apply_family(shhd_engine* e, int family) {
    check_cuda(cudaStreamSynchronize(e->stream), "stream synchronize");
    drop_graphs(e);
    e->family_override = family;
    e->pair_path = e->col_fixed = e->row_fixed = e->reg_row = e->split_row = e->dual_row = false;
    build_plan(e);
    // the split row pass's physical-row buffer exists only while that family is selected
    if (e->split_row && !e->phys) {
        e->phys_bytes = split_phys_member_elems(e->P) * e->cfg.batch * 16;
        e->phys = dalloc(e, e->phys_bytes);
    } else if (!e->split_row && e->phys) {
        cudaFree(e->phys);
        e->phys = nullptr;
        e->device_bytes -= e->phys_bytes;
        e->phys_bytes = 0;
    }
    for (void* p : {e->tw_x, e->tw_y})
        if (p) cudaFree(p);
    e->device_bytes -= e->tw_bytes;
    const auto twx = host_twiddles<T>(e, e->cfg.nx, e->row_fixed);
    const auto twy = host_twiddles<T>(e, e->cfg.ny, e->col_fixed);
    e->tw_x = dalloc(e, twx.size());
    e->tw_y = dalloc(e, twy.size());
    e->tw_bytes = twx.size() + twy.size();
    check_cuda(cudaMemcpyAsync(e->tw_x, twx.data(), twx.size(), cudaMemcpyHostToDevice, e->stream), "twiddle upload");
    check_cuda(cudaMemcpyAsync(e->tw_y, twy.data(), twy.size(), cudaMemcpyHostToDevice, e->stream), "twiddle upload");
    set_smem_attrs<T>(e);
    check_cuda(cudaStreamSynchronize(e->stream), "family sync");
}

template <typename T>
void autotune(shhd_engine* e, int trial_steps, int* family_out, int* chunk_out, double* ms_out) {
    if (trial_steps < 1) throw Failure(SHHD_EINVAL, "trial_steps must be positive");
    if (e->cfg.noise_source == SHHD_NOISE_EXTERNAL) throw Failure(SHHD_EINVAL, "autotune needs Philox noise (external noise steps one at a time)");
    check_cuda(cudaStreamSynchronize(e->stream), "stream synchronize");
    const size_t bytes = e->state_elems * e->cfg.batch * sizeof(cplx<T>);
    const size_t k0b = e->k0_u ? sizeof(double2) * e->cfg.batch * e->P.nfields : 0;
    void* save = nullptr;
    void* save_k0 = nullptr;
    check_cuda(cudaMalloc(&save, bytes), "autotune save buffer");
    if (k0b) check_cuda(cudaMalloc(&save_k0, k0b), "autotune save buffer");
    // device buffers the per-stage measure taps accumulate into while trials step: saved with the
    // state and restored after every trial, so that a measure's sums hold no trial steps
    struct Kept { void* dev; size_t bytes; void* copy; };
    std::vector<Kept> kept;
    const size_t B = e->cfg.batch;
    if (e->gk_on) {
        const GkArgs& G = e->gk;
        kept.push_back({G.sums, sizeof(double) * B * G.ntau * G.nmodes, nullptr});
        kept.push_back({G.integral, sizeof(double2) * B * G.nmodes, nullptr});
        kept.push_back({G.flux_step, sizeof(double2) * B * G.nmodes, nullptr});
    }
    if (e->flux0_on) kept.push_back({e->flux0.acc, sizeof(double) * B * e->flux0.ncol, nullptr});
    for (int ax = 0; ax < 2; ++ax)
        if (e->fline_on[ax]) kept.push_back({e->fline[ax].acc, sizeof(double2) * B * e->fline[ax].ncomp * e->fline[ax].nline, nullptr});
    auto free_kept = [&] {
        for (Kept& k : kept)
            if (k.copy) cudaFree(k.copy);
    };
    cudaEvent_t a = nullptr, b = nullptr;
    const int64_t step0 = e->step_index;
    const double time0 = e->time;
    const int64_t l0[4] = {e->kernel_launches[0], e->kernel_launches[1], e->kernel_launches[2], e->kernel_launches[3]};
    const double b0[4] = {e->kernel_bytes[0], e->kernel_bytes[1], e->kernel_bytes[2], e->kernel_bytes[3]};
    const bool prof = e->profiling;
    e->profiling = false;
    auto restore = [&] {
        check_cuda(cudaMemcpyAsync(e->u, save, bytes, cudaMemcpyDeviceToDevice, e->stream), "autotune restore");
        if (k0b) check_cuda(cudaMemcpyAsync(e->k0_u, save_k0, k0b, cudaMemcpyDeviceToDevice, e->stream), "autotune restore");
        for (const Kept& k : kept) check_cuda(cudaMemcpyAsync(k.dev, k.copy, k.bytes, cudaMemcpyDeviceToDevice, e->stream), "autotune restore");
        e->step_index = step0;
        e->time = time0;
    };
    try {
        check_cuda(cudaMemcpyAsync(save, e->u, bytes, cudaMemcpyDeviceToDevice, e->stream), "autotune save");
        if (k0b) check_cuda(cudaMemcpyAsync(save_k0, e->k0_u, k0b, cudaMemcpyDeviceToDevice, e->stream), "autotune save");
        for (Kept& k : kept) {
            check_cuda(cudaMalloc(&k.copy, k.bytes), "autotune save buffer");
            check_cuda(cudaMemcpyAsync(k.copy, k.dev, k.bytes, cudaMemcpyDeviceToDevice, e->stream), "autotune save");
        }
        check_cuda(cudaEventCreate(&a), "cudaEventCreate");
        check_cuda(cudaEventCreate(&b), "cudaEventCreate");
        // candidates: kernel families valid for this configuration x {direct launches, one graph of trial_steps}
        std::vector<int> families = {0};
        {
            shhd_engine probe = *e;  // host copy for planning only: is the pair-line family valid here?
            probe.family_override = 1;
            probe.pair_path = probe.col_fixed = probe.row_fixed = false;
            build_plan(&probe);
            if (probe.pair_path) families.push_back(1);
            probe.family_override = 2;
            probe.pair_path = probe.col_fixed = probe.row_fixed = probe.reg_row = false;
            build_plan(&probe);
            if (probe.reg_row && e->tw_reg) families.push_back(2);
            probe.family_override = 3;
            probe.pair_path = probe.col_fixed = probe.row_fixed = probe.reg_row = probe.split_row = false;
            build_plan(&probe);
            if (probe.split_row) families.push_back(3);
            probe.family_override = 4;
            probe.pair_path = probe.col_fixed = probe.row_fixed = probe.reg_row = probe.split_row = probe.dual_row = false;
            build_plan(&probe);
            if (probe.dual_row) families.push_back(4);
        }
        int chunk_trial = trial_steps;
        if (e->cfg.integrator == SHHD_EULER && chunk_trial % 2) ++chunk_trial;
        // ms per step of chunk_trial steps after as many untimed ones (warm-up and capture), from the saved state
        auto trial = [&] {
            drop_graphs(e);
            enqueue(e, chunk_trial);
            check_cuda(cudaEventRecord(a, e->stream), "cudaEventRecord");
            enqueue(e, chunk_trial);
            check_cuda(cudaEventRecord(b, e->stream), "cudaEventRecord");
            sync_and_check(e);
            float ms = 0.f;
            check_cuda(cudaEventElapsedTime(&ms, a, b), "cudaEventElapsedTime");
            restore();
            return ms / chunk_trial;
        };
        // families at the rule's launch shapes
        e->row_blocks = e->col_blocks = 0;
        double best = 1e300;
        int best_family = 0, best_chunk = 0, idx = 0;
        for (int fam : families) {
            apply_family<T>(e, fam);
            for (int chunk : {0, chunk_trial}) {
                e->graph_chunk = chunk;
                const double per = trial();
                if (ms_out) ms_out[idx] = per;
                ++idx;
                if (per < best) { best = per; best_family = fam; best_chunk = chunk; }
            }
        }
        drop_graphs(e);
        apply_family<T>(e, best_family);
        e->graph_chunk = best_chunk;
        // then the launch shapes of the chosen family's pair-line kernels: registers for three or
        // two row-pass blocks per SM where shared memory holds three, for four or three
        // column-forward blocks on >= 384-point columns where it holds four
        std::vector<int> rows = {0}, cols = {0};
        if (pair_line_row(e) && e->smem_row <= kRowThreeBlockSmem) rows = {2, 3};
        if (e->pair_path && e->P.n_groups > 0 && e->P.npy >= 384 && e->smem_col <= kColFourBlockSmem) cols = {3, 4};
        if (rows.size() * cols.size() > 1) {
            double best_shape = 1e300;
            int best_row = 0, best_col = 0;
            for (int r : rows)
                for (int c : cols) {
                    e->row_blocks = r;
                    e->col_blocks = c;
                    const double per = trial();
                    if (per < best_shape) { best_shape = per; best_row = r; best_col = c; }
                }
            e->row_blocks = best_row;
            e->col_blocks = best_col;
            drop_graphs(e);
        }
        if (family_out) *family_out = best_family;
        if (chunk_out) *chunk_out = best_chunk;
    } catch (...) {
        e->profiling = prof;
        cudaStreamSynchronize(e->stream);
        cudaFree(save);
        if (save_k0) cudaFree(save_k0);
        free_kept();
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
        throw;
    }
    restore();
    check_cuda(cudaStreamSynchronize(e->stream), "autotune sync");
    for (int k = 0; k < 4; ++k) { e->kernel_launches[k] = l0[k]; e->kernel_bytes[k] = b0[k]; }
    e->profiling = prof;
    cudaFree(save);
    if (save_k0) cudaFree(save_k0);
    free_kept();
    cudaEventDestroy(a);
    cudaEventDestroy(b);
}

}  // namespace

extern "C" {

int shhd_engine_autotune(shhd_engine* e, int trial_steps, int* family, int* graph_chunk, double* ms_per_step) {
    return guarded([&] {
        if (!e) throw Failure(SHHD_EINVAL, "null engine");
        check_cuda(cudaSetDevice(e->device), "cudaSetDevice");
        if (e->fp32) autotune<float>(e, trial_steps, family, graph_chunk, ms_per_step);
        else autotune<double>(e, trial_steps, family, graph_chunk, ms_per_step);
    });
}

}  // extern "C"

namespace {

// device spec of a C-ABI initial-field description, with its style's checks (the reference's
// parse-time and apply-time errors, in its words)
IcSpec resolve_initial_field(shhd_engine* e, const shhd_initial_field& in) {
    const StepPlan& P = e->P;
    const double ng = static_cast<double>(e->cfg.nx) * e->cfg.ny;
    constexpr double PI = 3.14159265358979323846;
    IcSpec s{};
    s.style = in.style;
    s.channel = in.channel;
    s.seed = in.seed;
    s.mean = in.mean;
    s.s0 = in.s0; s.c0 = in.c0; s.c2 = in.c2; s.c4 = in.c4;
    s.n0 = in.n0; s.sigma = in.sigma;
    s.x0 = in.x0; s.y0 = in.y0; s.sx = in.sigma_x; s.sy = in.sigma_y;
    s.nkx = in.nkx; s.nky = in.nky;
    s.lx = e->cfg.lx; s.ly = e->cfg.ly;
    auto each_active_k2 = [&](auto&& f) {
        for (int gx = 0; gx < P.hx; ++gx)
            for (int j = 0; j < P.kyn; ++j) {
                const int ky = j < P.nay / 2 ? j : j - P.kyn;
                if (gx == 0 && ky == 0) continue;
                const double kx = 2.0 * PI * gx / s.lx, kyv = 2.0 * PI * ky / s.ly;
                f(kx * kx + kyv * kyv);
            }
    };
    switch (in.style) {
        case SHHD_IC_GAUSSIAN_MODES:
            if (in.s0 < 0.0) throw Failure(SHHD_EINVAL, "the variance scale must be nonnegative");
            if (in.s0 != 0.0)  // initial_condition_equilibrium_gaussian_order_parameter.cc: positive coefficient on every active k != 0
                each_active_k2([&](double k2) {
                    if (!(in.c0 + in.c2 * k2 + in.c4 * k2 * k2 > 0.0))
                        throw Failure(SHHD_EINVAL, "set order_parameter equilibrium/gaussian requires positive linear chemical-potential "
                                                   "coefficient for every active nonzero mode.");
                });
            break;
        case SHHD_IC_TRANSVERSE_GAUSSIAN:
            if (in.s0 < 0.0) throw Failure(SHHD_EINVAL, "the variance scale must be nonnegative");
            if (in.channel != 0 && in.channel != 1) throw Failure(SHHD_EINVAL, "direction must be 0 or 1");
            break;
        case SHHD_IC_RANDOM_VORTICITY:
            if (in.channel != 0 && in.channel != 1) throw Failure(SHHD_EINVAL, "direction must be 0 or 1");
            if (!(in.n0 > 0.0)) throw Failure(SHHD_EINVAL, "set momentum random_vorticity requires positive n0.");
            if (!(in.sigma > 0.0)) throw Failure(SHHD_EINVAL, "set momentum random_vorticity requires positive sigma.");
            if (!(in.amplitude > 0.0)) throw Failure(SHHD_EINVAL, "set momentum random_vorticity requires positive urms.");
            break;  // factor: from the device norm
        case SHHD_IC_BUMP:
            if (!(in.sigma_x > 0.0) || !(in.sigma_y > 0.0)) throw Failure(SHHD_EINVAL, "gaussian requires positive sigma values");
            s.factor = in.amplitude * ng * 2.0 * PI * in.sigma_x * in.sigma_y / (s.lx * s.ly);
            break;
        case SHHD_IC_SINE:
            if (in.nkx < 0 || in.nkx >= P.hx) throw Failure(SHHD_EINVAL, "sine requires 0 <= nkx < Nx/2; Nyquist line is fixed to zero");
            if (in.nky <= -(P.nay / 2) || in.nky >= P.nay / 2)
                throw Failure(SHHD_EINVAL, "sine requires -Ny/2 < nky < Ny/2; Nyquist line is fixed to zero");
            if (in.nkx == 0 && in.nky == 0) throw Failure(SHHD_EINVAL, "sine requires a nonzero wave number");
            s.factor = -0.5 * in.amplitude * ng;
            break;
        default: throw Failure(SHHD_EINVAL, "unknown initial-field style " + std::to_string(in.style));
    }
    if (in.style == SHHD_IC_RANDOM_VORTICITY) {
        // initial_condition_random_vorticity_momentum.cc:108-131: the norm of the unnormalised shell over both
        // components, summed on the device in a fixed order
        const int nblk = static_cast<int>((static_cast<size_t>(P.hx) * P.kyn + kThreads - 1) / kThreads);
        const size_t need = sizeof(double) * (static_cast<size_t>(nblk) + 1);
        if (e->ic_scratch_bytes < need) {
            if (e->ic_scratch) { check_cuda(cudaFree(e->ic_scratch), "cudaFree"); e->device_bytes -= e->ic_scratch_bytes; e->ic_scratch = nullptr; }
            e->ic_scratch = static_cast<double*>(dalloc(e, need));
            e->ic_scratch_bytes = need;
        }
        vorticity_norm_kernel<<<nblk, kThreads, 0, e->stream>>>(P, s, e->ic_scratch + 1);
        check_cuda(cudaGetLastError(), "vorticity_norm launch");
        sum_partials_kernel<<<1, kThreads, 0, e->stream>>>(e->ic_scratch + 1, nblk, 1, e->ic_scratch);
        check_cuda(cudaGetLastError(), "sum_partials launch");
        double norm = 0.0;
        check_cuda(cudaMemcpyAsync(&norm, e->ic_scratch, sizeof(double), cudaMemcpyDeviceToHost, e->stream), "norm read");
        check_cuda(cudaStreamSynchronize(e->stream), "norm sync");
        if (norm == 0.0) throw Failure(SHHD_EINVAL, "set momentum random_vorticity generated zero velocity field.");
        if (in.rho0 == 0.0) throw Failure(SHHD_EINVAL, "set momentum random_vorticity requires nonzero reference density.");
        const double scale = in.amplitude * ng / std::sqrt(norm);
        s.factor = in.rho0 * scale;
    }
    return s;
}

}  // namespace

extern "C" {

int shhd_engine_set_initial_field(shhd_engine* e, int member, int field, const shhd_initial_field* spec) {
    return guarded([&] {
        if (!e || !spec) throw Failure(SHHD_EINVAL, "null argument");
        if (member < 0 || member >= e->cfg.batch) throw Failure(SHHD_EINVAL, "member index out of range");
        if (field < 0 || field >= e->P.nfields) throw Failure(SHHD_EINVAL, "field index out of range");
        check_cuda(cudaSetDevice(e->device), "cudaSetDevice");
        const IcSpec s = resolve_initial_field(e, *spec);
        const StepPlan& P = e->P;
        const size_t modes = static_cast<size_t>(P.hx) * P.kyn;
        const dim3 g(static_cast<unsigned>((modes + kThreads - 1) / kThreads));
        double2* k0 = e->k0_u ? e->k0_u + static_cast<size_t>(member) * P.nfields + field : nullptr;
        if (e->fp32)
            initial_field_kernel<float><<<g, kThreads, 0, e->stream>>>(P, static_cast<float2*>(e->u), member, field, s, k0);
        else
            initial_field_kernel<double><<<g, kThreads, 0, e->stream>>>(P, static_cast<double2*>(e->u), member, field, s, k0);
        check_cuda(cudaGetLastError(), "initial_field launch");
        double2 v00{};  // the density's (0, 0) coefficient in FP64 (FP32 engines' copy, else the state), as set_state takes it
        if (field == 0) {
            const void* src = k0 ? static_cast<const void*>(k0)
                                 : static_cast<const void*>(static_cast<const double2*>(e->u) + static_cast<size_t>(member) * P.nfields * modes);
            check_cuda(cudaMemcpyAsync(&v00, src, sizeof(double2), cudaMemcpyDeviceToHost, e->stream), "k = 0 read");
        }
        check_cuda(cudaStreamSynchronize(e->stream), "initial_field sync");
        if (field == 0) e->rho0_candidate[member] = v00.x / (static_cast<double>(e->cfg.nx) * e->cfg.ny);
    });
}

int shhd_engine_check_transverse(shhd_engine* e, const shhd_initial_field* jx, const shhd_initial_field* jy) {
    return guarded([&] {
        if (!e || !jx || !jy) throw Failure(SHHD_EINVAL, "null argument");
        check_cuda(cudaSetDevice(e->device), "cudaSetDevice");
        const IcSpec sx = resolve_initial_field(e, *jx), sy = resolve_initial_field(e, *jy);
        if (!e->flag_dev) e->flag_dev = static_cast<int*>(dalloc(e, sizeof(int)));
        check_cuda(cudaMemsetAsync(e->flag_dev, 0, sizeof(int), e->stream), "flag clear");
        const StepPlan& P = e->P;
        const size_t modes = static_cast<size_t>(P.hx) * P.kyn;
        transverse_check_kernel<<<static_cast<unsigned>((modes + kThreads - 1) / kThreads), kThreads, 0, e->stream>>>(P, sx, sy, e->flag_dev);
        check_cuda(cudaGetLastError(), "transverse_check launch");
        int bad = 0;
        check_cuda(cudaMemcpyAsync(&bad, e->flag_dev, sizeof(int), cudaMemcpyDeviceToHost, e->stream), "flag read");
        check_cuda(cudaStreamSynchronize(e->stream), "transverse_check sync");
        if (bad)
            throw Failure(SHHD_EINVAL, "incompressible initial momentum must be transverse: k dot j must be zero for every nonzero active "
                                       "spectral mode.");
    });
}

int shhd_engine_set_gaussian_field(shhd_engine* e, int member, int field, uint64_t seed, int channel, double mean, double s0, double c0,
                                   double c2, double c4) {
    shhd_initial_field spec{};
    spec.style = SHHD_IC_GAUSSIAN_MODES;
    spec.channel = channel;
    spec.seed = seed;
    spec.mean = mean;
    spec.s0 = s0; spec.c0 = c0; spec.c2 = c2; spec.c4 = c4;
    return shhd_engine_set_initial_field(e, member, field, &spec);
}

}  // extern "C"

namespace {

// the measure plan: the step plan's geometry and physics with runtime-plan transforms
template <typename T>
void build_measure_plan(shhd_engine* e) {
    MeasurePlan& M = e->meas;
    if (M.ready) return;
    const shhd_config& c = e->cfg;
    const size_t cs = sizeof(cplx<T>);
    const size_t smem_cap = 227 * 1024;
    StepPlan P = e->P;
    P.batch = 1;
    P.n_out = 0;
    P.n_groups = 0;
    P.fy = make_fft_plan(c.ny);
    P.fx = make_fft_plan(c.nx);
    P.twy_count = kTwLo + P.fy.tw_hi_count;
    P.twx_count = kTwLo + P.fx.tw_hi_count;
    auto col_bytes = [&](int w) { return static_cast<size_t>(P.twy_count + 2L * w * c.ny) * cs; };
    int W = 8;
    while (W > 1 && (P.hx % W != 0 || col_bytes(W) > 100 * 1024)) W /= 2;
    if (col_bytes(W) > smem_cap) throw Failure(SHHD_EUNSUPPORTED, "energy measure: compute grid too large for the column transform");
    P.W = W;
    P.logw = W == 8 ? 3 : (W == 4 ? 2 : (W == 2 ? 1 : 0));
    P.ntiles = P.hx / W;
    P.fy.swz = swizzle_mask(c.ny, e->fp32 ? 16 : 8, W);
    P.fx.swz = swizzle_mask(c.nx, e->fp32 ? 16 : 8, 1);
    P.div_w = make_fastdiv(W);
    P.div_kyn = make_fastdiv(P.kyn);
    P.kyp = (P.kyn + 7) & ~7;
    P.div_kyp = make_fastdiv(P.kyp);
    P.div_npy = make_fastdiv(c.ny);
    P.div_hx = make_fastdiv(P.hx);
    // row pass: at most 3 input lines (every order parameter for a plugin style's density) and
    // row_lb ping-pong lines
    const int nin = std::max(3, c.free_energy == SHHD_FE_PLUGIN ? c.num_order_parameters : 0);
    const size_t line = static_cast<size_t>(c.nx) * cs;
    auto row_bytes = [&](int lb) { return static_cast<size_t>(P.twx_count) * cs + (nin + lb) * line; };
    int lb = 3;
    while (lb > 1 && row_bytes(lb) > 113 * 1024) --lb;
    if (row_bytes(lb) > smem_cap) throw Failure(SHHD_EUNSUPPORTED, "energy measure: compute grid too large for the row transform");
    P.row_lb = lb;
    P.row_nb = lb;
    M.P = P;
    M.smem_col = col_bytes(W);
    M.smem_row = row_bytes(lb);
    const auto twx = twiddle_table<T>(c.nx), twy = twiddle_table<T>(c.ny);
    M.tw_x = dalloc(e, twx.size() * cs);
    M.tw_y = dalloc(e, twy.size() * cs);
    check_cuda(cudaMemcpyAsync(M.tw_x, twx.data(), twx.size() * cs, cudaMemcpyHostToDevice, e->stream), "twiddle upload");
    check_cuda(cudaMemcpyAsync(M.tw_y, twy.data(), twy.size() * cs, cudaMemcpyHostToDevice, e->stream), "twiddle upload");
    M.i1 = dalloc(e, static_cast<size_t>(nin) * P.hx * c.ny * cs);
    MemberInfo mi{};
    mi.active = 1;
    M.member = dalloc(e, sizeof(MemberInfo));
    check_cuda(cudaMemcpyAsync(M.member, &mi, sizeof(MemberInfo), cudaMemcpyHostToDevice, e->stream), "member upload");
    const size_t nblk = (static_cast<size_t>(P.hx) * P.kyn + kThreads - 1) / kThreads;
    M.scratch_doubles = std::max(nblk * (2 + kMaxOp), static_cast<size_t>(c.ny / 2 + 1)) + 8 + kMaxOp;
    M.scratch = static_cast<double*>(dalloc(e, M.scratch_doubles * sizeof(double)));
    raise_smem_limit(reinterpret_cast<const void*>(col_inverse_kernel<T, 0>), M.smem_col);
    raise_smem_limit(reinterpret_cast<const void*>(energy_row_kernel<T>), M.smem_row);
    raise_smem_limit(reinterpret_cast<const void*>(profile_velocity_row_kernel<T>), M.smem_row);
    check_cuda(cudaStreamSynchronize(e->stream), "measure plan");
    M.ready = true;
}

// sum over the padded grid of one physical-space energy density (term 0 kinetic, 1 psi^4 of field f)
template <typename T>
double physical_energy_sum(shhd_engine* e, const cplx<T>* st, int term, int field) {
    MeasurePlan& M = e->meas;
    StepPlan P = M.P;
    if (term == 0) {
        P.n_in = 3;
        P.in_field[0] = 0;
        P.in_field[1] = P.nop + 1;
        P.in_field[2] = P.nop + 2;
    } else if (term == 2) {  // a plugin style's density: every order parameter
        P.n_in = P.nop;
        for (int a = 0; a < P.nop; ++a) P.in_field[a] = 1 + a;
    } else {
        P.n_in = 1;
        P.in_field[0] = field;
    }
    auto* i1 = static_cast<cplx<T>*>(M.i1);
    col_inverse_kernel<T, 0><<<dim3(P.ntiles, P.n_in, 1), kThreads, M.smem_col, e->stream>>>(
        P, static_cast<const MemberInfo*>(M.member), st, i1, static_cast<const cplx<T>*>(M.tw_y));
    check_cuda(cudaGetLastError(), "measure col_inverse launch");
    const int pairs = (P.npy + 1) / 2;
    energy_row_kernel<T><<<pairs, kThreads, M.smem_row, e->stream>>>(P, i1, static_cast<const cplx<T>*>(M.tw_x), term, M.scratch);
    check_cuda(cudaGetLastError(), "energy_row launch");
    double* out = M.scratch + M.scratch_doubles - 1;
    sum_partials_kernel<<<1, kThreads, 0, e->stream>>>(M.scratch, pairs, 1, out);
    check_cuda(cudaGetLastError(), "sum_partials launch");
    double v = 0.0;
    check_cuda(cudaMemcpyAsync(&v, out, sizeof(double), cudaMemcpyDeviceToHost, e->stream), "energy read");
    check_cuda(cudaStreamSynchronize(e->stream), "energy sync");
    return v;
}

// the spectral line of one field that a profile along `axis` needs (FP64)
template <typename T>
void profile_line(shhd_engine* e, int member, int field, int axis, double* out) {
    const StepPlan& P = e->P;
    const size_t fstride = static_cast<size_t>(P.hx) * P.kyn;
    const auto* f = static_cast<const cplx<T>*>(e->u) + static_cast<size_t>(member) * e->state_elems + field * fstride;
    const double2* k0 = e->k0_u ? e->k0_u + static_cast<size_t>(member) * P.nfields + field : nullptr;
    const int n = axis == 0 ? P.hx : P.kyn;
    MeasurePlan& M = e->meas;
    if (!M.line) M.line = static_cast<double2*>(dalloc(e, sizeof(double2) * std::max(P.hx, P.kyn)));
    profile_line_kernel<T><<<(n + kThreads - 1) / kThreads, kThreads, 0, e->stream>>>(P, f, k0, axis, M.line);
    check_cuda(cudaGetLastError(), "profile_line launch");
    check_cuda(cudaMemcpyAsync(out, M.line, sizeof(double2) * n, cudaMemcpyDeviceToHost, e->stream), "profile line read");
    check_cuda(cudaStreamSynchronize(e->stream), "profile sync");
}

// compressible velocity component of one member summed over the transverse axis
template <typename T>
void profile_velocity(shhd_engine* e, int member, int component, int axis, double* out) {
    build_measure_plan<T>(e);
    MeasurePlan& M = e->meas;
    StepPlan P = M.P;
    P.n_in = 3;
    P.in_field[0] = 0;
    P.in_field[1] = P.nop + 1;
    P.in_field[2] = P.nop + 2;
    const int pairs = (P.npy + 1) / 2;
    if (!M.profile) {
        M.profile = static_cast<double*>(dalloc(e, sizeof(double) * (static_cast<size_t>(pairs) * P.npx + std::max(P.npx, P.npy))));
        M.flag = static_cast<int*>(dalloc(e, sizeof(int)));
    }
    const auto* st = static_cast<const cplx<T>*>(e->u) + static_cast<size_t>(member) * e->state_elems;
    auto* i1 = static_cast<cplx<T>*>(M.i1);
    check_cuda(cudaMemsetAsync(M.flag, 0, sizeof(int), e->stream), "flag clear");
    col_inverse_kernel<T, 0><<<dim3(P.ntiles, P.n_in, 1), kThreads, M.smem_col, e->stream>>>(
        P, static_cast<const MemberInfo*>(M.member), st, i1, static_cast<const cplx<T>*>(M.tw_y));
    check_cuda(cudaGetLastError(), "measure col_inverse launch");
    double* res = M.profile + static_cast<size_t>(pairs) * P.npx;
    profile_velocity_row_kernel<T><<<pairs, kThreads, M.smem_row, e->stream>>>(P, i1, static_cast<const cplx<T>*>(M.tw_x), axis, component,
                                                                               axis == 0 ? M.profile : res, M.flag);
    check_cuda(cudaGetLastError(), "profile_velocity launch");
    if (axis == 0) {
        column_sums_kernel<<<(P.npx + kThreads - 1) / kThreads, kThreads, 0, e->stream>>>(M.profile, pairs, P.npx, res);
        check_cuda(cudaGetLastError(), "column_sums launch");
    }
    int bad = 0;
    const int n = axis == 0 ? P.npx : P.npy;
    check_cuda(cudaMemcpyAsync(out, res, sizeof(double) * n, cudaMemcpyDeviceToHost, e->stream), "profile read");
    check_cuda(cudaMemcpyAsync(&bad, M.flag, sizeof(int), cudaMemcpyDeviceToHost, e->stream), "flag read");
    check_cuda(cudaStreamSynchronize(e->stream), "profile sync");
    if (bad) throw Failure(SHHD_EINVAL, "AveProfileMeasure compressible velocity encountered zero density.");
}

// E_T, E_K, E_psi, E_C of one member (measure_time_series.cc:152-188, 305-470)
template <typename T>
void energies(shhd_engine* e, int member, double* out) {
    build_measure_plan<T>(e);
    MeasurePlan& M = e->meas;
    const StepPlan& P = e->P;
    const shhd_config& c = e->cfg;
    const int nop = P.nop;
    const double ng = static_cast<double>(c.nx) * c.ny, cell = c.lx * c.ly / ng;
    const auto* st = static_cast<const cplx<T>*>(e->u) + static_cast<size_t>(member) * e->state_elems;
    const double2* k0 = e->k0_u ? e->k0_u + static_cast<size_t>(member) * P.nfields : nullptr;
    // spectral sums
    const int nv = 2 + nop;
    const int nblk = static_cast<int>((static_cast<size_t>(P.hx) * P.kyn + kThreads - 1) / kThreads);
    double* sums = M.scratch + M.scratch_doubles - 1 - nv;
    energy_spectral_kernel<T><<<nblk, kThreads, 0, e->stream>>>(P, st, k0, M.scratch);
    check_cuda(cudaGetLastError(), "energy_spectral launch");
    sum_partials_kernel<<<nv, kThreads, 0, e->stream>>>(M.scratch, nblk, nv, sums);
    check_cuda(cudaGetLastError(), "sum_partials launch");
    std::vector<double> v(nv);
    check_cuda(cudaMemcpyAsync(v.data(), sums, sizeof(double) * nv, cudaMemcpyDeviceToHost, e->stream), "energy read");
    // rho(0, 0) in FP64: the FP32 engines' k = 0 copy (always allocated for them), else the FP64 state
    double2 rho00{};
    const void* src = k0 ? static_cast<const void*>(k0) : static_cast<const void*>(st);
    check_cuda(cudaMemcpyAsync(&rho00, src, sizeof(double2), cudaMemcpyDeviceToHost, e->stream), "rho(0) read");
    check_cuda(cudaStreamSynchronize(e->stream), "energy sync");
    const double rho0 = rho00.x / ng;
    const bool comp = c.mode == SHHD_COMPRESSIBLE, incomp = c.mode == SHHD_INCOMPRESSIBLE;
    double kin = 0.0, free_e = 0.0, compress = 0.0;
    if (comp) kin = physical_energy_sum<T>(e, st, 0, 0) * cell;
    else if (incomp) kin = 0.5 * cell / (ng * rho0) * v[0];
    if (comp && P.cT2 != 0.0) compress = 0.5 * P.cT2 * cell / (ng * rho0) * v[1];
    for (int a = 0; a < nop; ++a)
        if (P.mu_k0[a] != 0.0 || P.mu_k2[a] != 0.0 || P.mu_k4[a] != 0.0) free_e += 0.5 * cell / ng * v[2 + a];
    for (int a = 0; a < nop; ++a)
        if (P.mu_u3[a] != 0.0) free_e += 0.25 * P.mu_u3[a] * physical_energy_sum<T>(e, st, 1, 1 + a) * cell;
    if (P.fe_plugin && nop > 0) free_e += physical_energy_sum<T>(e, st, 2, 0) * cell;
    out[0] = kin + free_e + compress;
    out[1] = kin;
    out[2] = free_e;
    out[3] = compress;
}

}  // namespace

extern "C" {

int shhd_engine_energies(shhd_engine* e, int member, double* out, size_t n) {
    return guarded([&] {
        if (!e || !out) throw Failure(SHHD_EINVAL, "null argument");
        if (member < 0 || member >= e->cfg.batch) throw Failure(SHHD_EINVAL, "member index out of range");
        if (n < 4) throw Failure(SHHD_EINVAL, "energies need 4 doubles");
        check_cuda(cudaSetDevice(e->device), "cudaSetDevice");
        if (e->fp32) energies<float>(e, member, out);
        else energies<double>(e, member, out);
    });
}

int shhd_engine_profile_line(shhd_engine* e, int member, int field, int axis, double* out, size_t n) {
    return guarded([&] {
        if (!e || !out) throw Failure(SHHD_EINVAL, "null argument");
        if (member < 0 || member >= e->cfg.batch) throw Failure(SHHD_EINVAL, "member index out of range");
        if (field < 0 || field >= e->P.nfields) throw Failure(SHHD_EINVAL, "field index out of range");
        if (axis != 0 && axis != 1) throw Failure(SHHD_EINVAL, "ave/profile measure: axis must be x|y|0|1.");
        const size_t need = 2 * static_cast<size_t>(axis == 0 ? e->P.hx : e->P.kyn);
        if (n < need) throw Failure(SHHD_EINVAL, "profile line needs " + std::to_string(need) + " doubles");
        check_cuda(cudaSetDevice(e->device), "cudaSetDevice");
        if (e->fp32) profile_line<float>(e, member, field, axis, out);
        else profile_line<double>(e, member, field, axis, out);
    });
}

int shhd_engine_profile_velocity(shhd_engine* e, int member, int component, int axis, double* out, size_t n) {
    return guarded([&] {
        if (!e || !out) throw Failure(SHHD_EINVAL, "null argument");
        if (member < 0 || member >= e->cfg.batch) throw Failure(SHHD_EINVAL, "member index out of range");
        if (component != 0 && component != 1) throw Failure(SHHD_EINVAL, "component must be 0 (x) or 1 (y)");
        if (axis != 0 && axis != 1) throw Failure(SHHD_EINVAL, "ave/profile measure: axis must be x|y|0|1.");
        if (e->cfg.mode != SHHD_COMPRESSIBLE) throw Failure(SHHD_EINVAL, "the physical-space velocity profile is the compressible one");
        const size_t need = static_cast<size_t>(axis == 0 ? e->cfg.nx : e->cfg.ny);
        if (n < need) throw Failure(SHHD_EINVAL, "profile needs " + std::to_string(need) + " doubles");
        check_cuda(cudaSetDevice(e->device), "cudaSetDevice");
        if (e->fp32) profile_velocity<float>(e, member, component, axis, out);
        else profile_velocity<double>(e, member, component, axis, out);
    });
}

int shhd_engine_l2_sums(shhd_engine* e, int member, double* out, size_t n) {
    return guarded([&] {
        if (!e || !out) throw Failure(SHHD_EINVAL, "null argument");
        if (member < 0 || member >= e->cfg.batch) throw Failure(SHHD_EINVAL, "member index out of range");
        const int nf = e->P.nfields;
        if (n != static_cast<size_t>(2 * nf)) throw Failure(SHHD_EINVAL, "size mismatch: expected 2 * nfields = " + std::to_string(2 * nf));
        check_cuda(cudaSetDevice(e->device), "cudaSetDevice");
        if (!e->l2_dev) e->l2_dev = static_cast<double*>(dalloc(e, sizeof(double) * 2 * kMaxFields));
        check_cuda(cudaMemsetAsync(e->l2_dev, 0, sizeof(double) * 2 * nf, e->stream), "memset");
        const size_t modes = static_cast<size_t>(e->P.hx) * e->P.kyn;
        const dim3 g(static_cast<unsigned>((modes + kThreads - 1) / kThreads));
        if (e->fp32) l2_sums_kernel<float><<<g, kThreads, 0, e->stream>>>(e->P, static_cast<const float2*>(e->u), member, e->l2_dev);
        else l2_sums_kernel<double><<<g, kThreads, 0, e->stream>>>(e->P, static_cast<const double2*>(e->u), member, e->l2_dev);
        check_cuda(cudaGetLastError(), "l2_sums launch");
        check_cuda(cudaMemcpyAsync(out, e->l2_dev, sizeof(double) * 2 * nf, cudaMemcpyDeviceToHost, e->stream), "l2 download");
        check_cuda(cudaStreamSynchronize(e->stream), "l2 sync");
        // prefactor cell_area / grid_size (measure_time_series.cc:295-298, 262-275)
        const double np2 = static_cast<double>(e->cfg.nx) * e->cfg.ny;
        const double pref = e->cfg.lx * e->cfg.ly / np2 / np2;
        for (int q = 0; q < 2 * nf; ++q) out[q] *= pref;
    });
}

int shhd_engine_flux0_enable(shhd_engine* e) {
    return guarded([&] {
        if (!e) throw Failure(SHHD_EINVAL, "null engine");
        if (e->flux0_on) return;
        check_cuda(cudaSetDevice(e->device), "cudaSetDevice");
        const StepPlan& P = e->P;
        Flux0Args F{};
        F.ncol = 3 + 2 * P.nop;
        for (int c = 0; c < F.ncol; ++c) F.o[c] = -1;
        for (int o = 0; o < P.n_out; ++o) {
            const int k = P.out_kind[o], a = P.out_arg[o];
            if (k == OUT_PXX) F.o[0] = o;
            if (k == OUT_PXY) F.o[1] = o;
            if (k == OUT_PYY) F.o[2] = o;
            if (k == OUT_PSIVX) F.o[3 + 2 * a] = o;
            if (k == OUT_PSIVY) F.o[4 + 2 * a] = o;
        }
        // j_det records the linear pressure flux whenever it runs with cT^2 != 0 (fcalculator.cc:110-136)
        F.pressure = e->cfg.mode != SHHD_QUIESCENT && P.cT2 != 0.0;
        F.pair_layout = e->pair_path ? 1 : 0;
        F.period = 1;
        F.phase = 0;
        const size_t bytes = sizeof(double) * e->cfg.batch * F.ncol;
        F.acc = static_cast<double*>(dalloc(e, bytes));
        check_cuda(cudaMemsetAsync(F.acc, 0, bytes, e->stream), "memset");
        check_cuda(cudaStreamSynchronize(e->stream), "flux0 sync");
        e->flux0 = F;
        e->flux0_on = true;
        drop_graphs(e);  // captured graphs do not hold the tap yet
    });
}

int shhd_engine_flux_line_enable(shhd_engine* e, int axis) {
    return guarded([&] {
        if (!e) throw Failure(SHHD_EINVAL, "null engine");
        if (axis != 0 && axis != 1) throw Failure(SHHD_EINVAL, "ave/profile measure: axis must be x|y|0|1.");
        if (e->fline_on[axis]) return;
        const StepPlan& P = e->P;
        const bool noisy = P.noise_j || [&] { for (int a = 0; a < P.nop; ++a) if (P.noise_psi[a]) return true; return false; }();
        if (noisy && e->cfg.noise_source == SHHD_NOISE_EXTERNAL)
            throw Failure(SHHD_EUNSUPPORTED, "the flux buffer needs the engine's own noise draws (replayed noise gives only its divergence)");
        check_cuda(cudaSetDevice(e->device), "cudaSetDevice");
        FluxLineArgs L{};
        L.axis = axis;
        L.nline = axis == 0 ? P.hx : P.kyn;
        L.ncomp = 3 + 2 * P.nop;
        L.pair_layout = e->pair_path ? 1 : 0;
        L.o_vx = L.o_vy = L.o_pxx = L.o_pxy = L.o_pyy = -1;
        for (int a = 0; a < kMaxOp; ++a) L.o_mu[a] = L.o_px[a] = L.o_py[a] = -1;
        for (int o = 0; o < P.n_out; ++o) {
            const int k = P.out_kind[o], a = P.out_arg[o];
            if (k == OUT_VX) L.o_vx = o;
            if (k == OUT_VY) L.o_vy = o;
            if (k == OUT_PXX) L.o_pxx = o;
            if (k == OUT_PXY) L.o_pxy = o;
            if (k == OUT_PYY) L.o_pyy = o;
            if (k == OUT_MU) L.o_mu[a] = o;
            if (k == OUT_PSIVX) L.o_px[a] = o;
            if (k == OUT_PSIVY) L.o_py[a] = o;
        }
        // the reference's conditions (fcalculator.cc:86-150)
        const shhd_config& c = e->cfg;
        const bool has_visc = c.eta != 0.0 || c.zeta != 0.0;
        L.mom_on = c.mode != SHHD_QUIESCENT && (P.cT2 != 0.0 || has_visc || c.momentum_advection);
        L.pressure = L.mom_on && P.cT2 != 0.0;
        L.visc_comp = L.mom_on && has_visc && c.mode == SHHD_COMPRESSIBLE;
        L.visc_incomp = L.mom_on && c.mode == SHHD_INCOMPRESSIBLE && c.eta != 0.0;
        if (L.visc_comp && (L.o_vx < 0 || L.o_vy < 0)) throw Failure(SHHD_EUNSUPPORTED, "viscous flux planes missing");
        for (int a = 0; a < P.nop; ++a) {
            L.psi_on[a] = c.mobility[a] != 0.0 || c.order_parameter_advection;
            L.psi_lin[a] = c.mobility[a] != 0.0 && (P.mu_k0[a] != 0.0 || P.mu_k2[a] != 0.0 || P.mu_k4[a] != 0.0);
            if (c.mobility[a] == 0.0) L.o_mu[a] = -1;
        }
        L.noise_j = P.noise_j;
        L.incompressible = c.mode == SHHD_INCOMPRESSIBLE;
        L.period = 1;
        L.phase = 0;
        std::vector<double2> wt(P.npy);
        for (int n = 0; n < P.npy; ++n) {
            const double ang = -2.0 * M_PI * n / P.npy;
            wt[n] = make_double2(std::cos(ang), std::sin(ang));
        }
        if (axis == 1) raise_smem_limit(reinterpret_cast<const void*>(e->fp32 ? reinterpret_cast<const void*>(flux_line_tap_kernel<float>)
                                                                                : reinterpret_cast<const void*>(flux_line_tap_kernel<double>)),
                                         sizeof(double2) * P.npy);
        L.wtab = static_cast<const double2*>(dalloc(e, sizeof(double2) * P.npy));
        check_cuda(cudaMemcpyAsync(const_cast<double2*>(L.wtab), wt.data(), sizeof(double2) * P.npy, cudaMemcpyHostToDevice, e->stream), "upload");
        const size_t bytes = sizeof(double2) * e->cfg.batch * L.ncomp * L.nline;
        L.acc = static_cast<double2*>(dalloc(e, bytes));
        check_cuda(cudaMemsetAsync(L.acc, 0, bytes, e->stream), "memset");
        check_cuda(cudaStreamSynchronize(e->stream), "flux line sync");
        e->fline[axis] = L;
        e->fline_on[axis] = true;
        drop_graphs(e);  // captured graphs do not hold the tap yet
    });
}

int shhd_engine_flux_tap_schedule(shhd_engine* e, int tap, int64_t period, int64_t phase) {
    return guarded([&] {
        if (!e) throw Failure(SHHD_EINVAL, "null engine");
        if (period < 1) throw Failure(SHHD_EINVAL, "the tap period must be positive");
        long long* per = nullptr;
        long long* ph = nullptr;
        if (tap == 0 && e->flux0_on) { per = &e->flux0.period; ph = &e->flux0.phase; }
        if ((tap == 1 || tap == 2) && e->fline_on[tap - 1]) { per = &e->fline[tap - 1].period; ph = &e->fline[tap - 1].phase; }
        if (!per) throw Failure(SHHD_EINVAL, "tap " + std::to_string(tap) + " is not enabled");
        const long long p = period, q = ((phase % period) + period) % period;
        if (*per != p || *ph != q) {
            *per = p;
            *ph = q;
            drop_graphs(e);  // captured graphs hold the schedule as a launch argument
        }
    });
}

int shhd_engine_flux_line_read(shhd_engine* e, int axis, int member, double* out, size_t n) {
    return guarded([&] {
        if (!e || !out) throw Failure(SHHD_EINVAL, "null argument");
        if (axis != 0 && axis != 1) throw Failure(SHHD_EINVAL, "ave/profile measure: axis must be x|y|0|1.");
        if (!e->fline_on[axis]) throw Failure(SHHD_EINVAL, "the flux line tap of this axis is not enabled");
        if (member < 0 || member >= e->cfg.batch) throw Failure(SHHD_EINVAL, "member index out of range");
        const FluxLineArgs& L = e->fline[axis];
        const size_t cnt = static_cast<size_t>(L.ncomp) * L.nline;
        if (n < 2 * cnt) throw Failure(SHHD_EINVAL, "flux line read needs " + std::to_string(2 * cnt) + " doubles");
        check_cuda(cudaSetDevice(e->device), "cudaSetDevice");
        check_cuda(cudaMemcpyAsync(out, L.acc + static_cast<size_t>(member) * cnt, sizeof(double2) * cnt, cudaMemcpyDeviceToHost, e->stream),
                   "flux line read");
        check_cuda(cudaStreamSynchronize(e->stream), "flux line sync");
    });
}

int shhd_engine_flux0_read(shhd_engine* e, int member, double* out, size_t n) {
    return guarded([&] {
        if (!e || !out) throw Failure(SHHD_EINVAL, "null argument");
        if (!e->flux0_on) throw Failure(SHHD_EINVAL, "the k = 0 flux tap is not enabled");
        if (member < 0 || member >= e->cfg.batch) throw Failure(SHHD_EINVAL, "member index out of range");
        const int ncol = e->flux0.ncol;
        if (n < static_cast<size_t>(ncol)) throw Failure(SHHD_EINVAL, "flux0 read needs 3 + 2 * num_order_parameters doubles");
        check_cuda(cudaSetDevice(e->device), "cudaSetDevice");
        check_cuda(cudaMemcpyAsync(out, e->flux0.acc + static_cast<size_t>(member) * ncol, sizeof(double) * ncol, cudaMemcpyDeviceToHost,
                                   e->stream),
                   "flux0 read");
        check_cuda(cudaStreamSynchronize(e->stream), "flux0 sync");
        const double ng = static_cast<double>(e->cfg.nx) * e->cfg.ny;
        for (int c = 0; c < ncol; ++c) out[c] /= ng;
    });
}

int shhd_engine_gk_enable(shhd_engine* e, int nevery, int nblock, int selection) {
    return guarded([&] {
        if (!e) throw Failure(SHHD_EINVAL, "null engine");
        if (e->gk_on) throw Failure(SHHD_EINVAL, "the Green-Kubo measure is already enabled");
        if (nevery <= 0 || nblock <= 0) throw Failure(SHHD_EINVAL, "nevery and nblock must be positive");
        if (nblock % nevery != 0) throw Failure(SHHD_EINVAL, "nblock must be a multiple of nevery");
        if (!(e->cfg.kBT > 0.0)) throw Failure(SHHD_EINVAL, "YokotaGreenKuboMeasure requires positive kBT from fix noise.");
        if (e->cfg.mode == SHHD_QUIESCENT) throw Failure(SHHD_EUNSUPPORTED, "the Green-Kubo stress measure needs momentum dynamics (not quiescent)");
        if (e->cfg.noise_source == SHHD_NOISE_EXTERNAL) throw Failure(SHHD_EUNSUPPORTED, "the Green-Kubo measure needs the engine's own noise draws");
        if (selection != 0 && selection != 1) throw Failure(SHHD_EINVAL, "YokotaGreenKuboMeasure: mode must be diagonal|all.");
        const StepPlan& P = e->P;
        // wave numbers of measure_yokota_green_kubo.cc:42-96
        const int max_nx = std::max(0, e->cfg.active_nx / 2 - 1), max_ny = std::max(0, e->cfg.active_ny / 2 - 1);
        std::vector<int2> modes;
        if (selection == 0) {
            for (int n = 1; n <= std::min(max_nx, max_ny); ++n) modes.push_back(make_int2(n, n));
        } else {
            for (int n = 1; n <= max_ny; ++n) modes.push_back(make_int2(0, n));
            for (int nx = 1; nx <= max_nx; ++nx)
                for (int ny = -max_ny; ny <= max_ny; ++ny) modes.push_back(make_int2(nx, ny));
        }
        if (modes.empty()) throw Failure(SHHD_EINVAL, "YokotaGreenKuboMeasure: no active wave vector is selected.");
        if (static_cast<double>(modes.size()) * P.npy > 64.0 * 1024 * 1024)
            throw Failure(SHHD_EUNSUPPORTED, "too many Green-Kubo modes for the direct column transforms at this grid (use diagonal)");
        check_cuda(cudaSetDevice(e->device), "cudaSetDevice");
        GkArgs& G = e->gk;
        G.nmodes = static_cast<int>(modes.size());
        G.nevery = nevery;
        G.nblock = nblock;
        G.ntau = nblock / nevery;
        G.kbt = e->cfg.kBT;
        G.area = e->cfg.lx * e->cfg.ly;
        G.cell_area = G.area / (static_cast<double>(e->cfg.nx) * e->cfg.ny);
        G.o_pxy = G.o_vx = G.o_vy = -1;
        for (int o = 0; o < P.n_out; ++o) {
            if (P.out_kind[o] == OUT_PXY) G.o_pxy = o;
            if (P.out_kind[o] == OUT_VX) G.o_vx = o;
            if (P.out_kind[o] == OUT_VY) G.o_vy = o;
        }
        G.pair_layout = e->pair_path ? 1 : 0;
        G.incomp_visc = P.incomp_visc;
        const size_t B = e->cfg.batch, nm = modes.size();
        std::vector<double2> wt(P.npy);
        for (int n = 0; n < P.npy; ++n) {
            const double a = -2.0 * M_PI * n / P.npy;
            wt[n] = make_double2(std::cos(a), std::sin(a));
        }
        G.modes = static_cast<const int2*>(dalloc(e, sizeof(int2) * nm));
        G.flux_step = static_cast<double2*>(dalloc(e, sizeof(double2) * B * nm));
        G.integral = static_cast<double2*>(dalloc(e, sizeof(double2) * B * nm));
        G.sums = static_cast<double*>(dalloc(e, sizeof(double) * B * G.ntau * nm));
        G.wtab = static_cast<const double2*>(dalloc(e, sizeof(double2) * P.npy));
        check_cuda(cudaMemcpyAsync(const_cast<int2*>(G.modes), modes.data(), sizeof(int2) * nm, cudaMemcpyHostToDevice, e->stream), "gk upload");
        check_cuda(cudaMemcpyAsync(const_cast<double2*>(G.wtab), wt.data(), sizeof(double2) * P.npy, cudaMemcpyHostToDevice, e->stream), "gk upload");
        check_cuda(cudaMemsetAsync(G.flux_step, 0, sizeof(double2) * B * nm, e->stream), "memset");
        check_cuda(cudaMemsetAsync(G.integral, 0, sizeof(double2) * B * nm, e->stream), "memset");
        check_cuda(cudaMemsetAsync(G.sums, 0, sizeof(double) * B * G.ntau * nm, e->stream), "memset");
        check_cuda(cudaStreamSynchronize(e->stream), "gk sync");
        e->gk_modes = modes;
        e->gk_sample_base.assign(B, 0);
        for (size_t m = 0; m < B; ++m) e->gk_sample_base[m] = (e->step_index - e->members[m].step0) / nblock;
        e->gk_on = true;
        drop_graphs(e);  // captured graphs do not hold the taps yet
    });
}

int shhd_engine_gk_read(shhd_engine* e, int member, double* sums, size_t n, int64_t* nsample, int reset) {
    return guarded([&] {
        if (!e || !sums) throw Failure(SHHD_EINVAL, "null argument");
        if (!e->gk_on) throw Failure(SHHD_EINVAL, "the Green-Kubo measure is not enabled");
        if (member < 0 || member >= e->cfg.batch) throw Failure(SHHD_EINVAL, "member index out of range");
        const GkArgs& G = e->gk;
        const size_t per = static_cast<size_t>(G.ntau) * G.nmodes;
        if (n != per) throw Failure(SHHD_EINVAL, "size mismatch: expected ntau * nmodes = " + std::to_string(per));
        check_cuda(cudaSetDevice(e->device), "cudaSetDevice");
        double* src = G.sums + static_cast<size_t>(member) * per;
        check_cuda(cudaMemcpyAsync(sums, src, per * sizeof(double), cudaMemcpyDeviceToHost, e->stream), "gk download");
        if (reset) check_cuda(cudaMemsetAsync(src, 0, per * sizeof(double), e->stream), "gk reset");
        check_cuda(cudaStreamSynchronize(e->stream), "gk sync");
        const int64_t done = (e->step_index - e->members[member].step0) / G.nblock;
        if (nsample) *nsample = done - e->gk_sample_base[member];
        if (reset) e->gk_sample_base[member] = done;
    });
}

int shhd_engine_set_family(shhd_engine* e, int family) {
    return guarded([&] {
        if (!e) throw Failure(SHHD_EINVAL, "null engine");
        if (family < -1 || family > 4) throw Failure(SHHD_EINVAL, "kernel family must be -1, 0, 1, 2, 3 or 4");
        check_cuda(cudaSetDevice(e->device), "cudaSetDevice");
        if (e->fp32) apply_family<float>(e, family);
        else apply_family<double>(e, family);
    });
}

int shhd_engine_family(const shhd_engine* e) {
    if (!e) return -1;
    return e->dual_row ? 4 : (e->split_row ? 3 : (e->reg_row ? 2 : (e->pair_path ? 1 : 0)));
}

int shhd_engine_set_launch_shape(shhd_engine* e, int row_blocks, int col_blocks) {
    return guarded([&] {
        if (!e) throw Failure(SHHD_EINVAL, "null engine");
        if (row_blocks != 0 && row_blocks != 2 && row_blocks != 3) throw Failure(SHHD_EINVAL, "row-pass blocks per SM must be 0, 2 or 3");
        if (col_blocks != 0 && col_blocks != 3 && col_blocks != 4)
            throw Failure(SHHD_EINVAL, "column-forward blocks per SM must be 0, 3 or 4");
        check_cuda(cudaSetDevice(e->device), "cudaSetDevice");
        check_cuda(cudaStreamSynchronize(e->stream), "stream synchronize");
        drop_graphs(e);
        e->row_blocks = row_blocks;
        e->col_blocks = col_blocks;
    });
}

int shhd_engine_launch_shape(const shhd_engine* e, int* row_blocks, int* col_blocks) {
    return guarded([&] {
        if (!e) throw Failure(SHHD_EINVAL, "null engine");
        if (row_blocks) *row_blocks = pair_line_row(e) ? (row_three_blocks(e) ? 3 : 2) : 0;
        if (col_blocks) *col_blocks = e->pair_path && e->P.n_groups > 0 ? (e->P.npy >= 384 ? (col_four_blocks(e) ? 4 : 3) : 2) : 0;
    });
}

int shhd_engine_set_graph_chunk(shhd_engine* e, int chunk) {
    return guarded([&] {
        if (!e) throw Failure(SHHD_EINVAL, "null engine");
        if (chunk < 0) throw Failure(SHHD_EINVAL, "graph chunk must be nonnegative");
        // Euler swaps its two state buffers every step: a replayed chunk must hold an even number of steps
        if (chunk > 0 && e->cfg.integrator == SHHD_EULER && chunk % 2) ++chunk;
        check_cuda(cudaSetDevice(e->device), "cudaSetDevice");
        check_cuda(cudaStreamSynchronize(e->stream), "stream synchronize");
        drop_graphs(e);
        e->graph_chunk = chunk;
    });
}

int shhd_engine_set_time(shhd_engine* e, int64_t step_index, double time) {
    if (!e) { g_last_error = "null engine"; return SHHD_EINVAL; }
    e->step_index = step_index;
    e->time = time;
    return SHHD_OK;
}

void* shhd_engine_stream(shhd_engine* e) { return e ? static_cast<void*>(e->stream) : nullptr; }

int shhd_engine_set_profiling(shhd_engine* e, int on) {
    return guarded([&] {
        if (!e) throw Failure(SHHD_EINVAL, "null engine");
        check_cuda(cudaStreamSynchronize(e->stream), "stream synchronize");
        resolve_timings(e);
        e->profiling = on != 0;
    });
}

int shhd_engine_kernel_stats(shhd_engine* e, double* total_ms, int64_t* launches, double* bytes) {
    return guarded([&] {
        if (!e) throw Failure(SHHD_EINVAL, "null engine");
        check_cuda(cudaStreamSynchronize(e->stream), "stream synchronize");
        resolve_timings(e);
        for (int k = 0; k < 4; ++k) {
            if (total_ms) total_ms[k] = e->kernel_ms[k];
            if (launches) launches[k] = e->kernel_launches[k];
            if (bytes) bytes[k] = e->kernel_bytes[k];
        }
    });
}

int shhd_engine_reset_stats(shhd_engine* e) {
    return guarded([&] {
        if (!e) throw Failure(SHHD_EINVAL, "null engine");
        check_cuda(cudaStreamSynchronize(e->stream), "stream synchronize");
        resolve_timings(e);
        for (int k = 0; k < 4; ++k) { e->kernel_ms[k] = 0; e->kernel_launches[k] = 0; e->kernel_bytes[k] = 0; }
    });
}

const void* shhd_engine_state_device(const shhd_engine* e) { return e ? e->u : nullptr; }

}  // extern "C"

// ---------------------------------------------------------------------------
// Right-hand side without device allocation
//
// For hosts that may not call cudaMalloc themselves: a solver embedded in a
// framework whose caching allocator owns the device memory (a second
// allocator would fragment it or exceed its budget), or a plugin loaded into
// a process whose memory was reserved up front.  They hand in device buffers
// they already own; every intermediate (column-inverse and product planes,
// the active-mode copies of input and output, twiddles, flags) lives in one
// fixed array compiled into this library.  That array is held on every GPU
// the library is loaded on, until the process exits.
// ---------------------------------------------------------------------------
namespace {

constexpr size_t kNoAllocAlign = 256;
static __device__ __align__(256) unsigned char g_noalloc_scratch[SHHD_NOALLOC_SCRATCH_BYTES];

// device address of the scratch array on the current device, looked up on every
// call (cheap beside the call's two stream waits), so a context created anew
// after cudaDeviceReset is never handed a stale address; the array's host-side
// name is not a device address
unsigned char* noalloc_base() {
    void* p = nullptr;
    check_cuda(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress of the static scratch");
    return static_cast<unsigned char*>(p);
}

// carves aligned regions out of the scratch array; sizes only, when base is null
struct ScratchCarver {
    unsigned char* base;
    size_t used = 0;
    void* take(size_t bytes) {
        void* p = base ? base + used : nullptr;
        used += (std::max<size_t>(bytes, 1) + kNoAllocAlign - 1) / kNoAllocAlign * kNoAllocAlign;
        return p;
    }
};

void check_device_buffer(const void* p, int device, const char* what) {
    if (!p) throw Failure(SHHD_EINVAL, std::string(what) + " is null");
    if (reinterpret_cast<uintptr_t>(p) % 16 != 0) throw Failure(SHHD_EINVAL, std::string(what) + " must be 16-byte aligned");
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        throw Failure(SHHD_EINVAL, std::string(what) + " is not a CUDA pointer");
    }
    if (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged)
        throw Failure(SHHD_EINVAL, std::string(what) + " must be device memory");
    if (a.type == cudaMemoryTypeDevice && a.device != device)
        throw Failure(SHHD_EINVAL, std::string(what) + " belongs to another device than the current one");
}

template <typename T>
void rhs_noalloc(shhd_engine* e, const double* state_dev, double* rhs_dev, unsigned char* base) {
    const StepPlan& P = e->P;
    const size_t cs = sizeof(cplx<T>);
    const auto twx = host_twiddles<T>(e, e->cfg.nx, e->row_fixed);
    const auto twy = host_twiddles<T>(e, e->cfg.ny, e->col_fixed);
    ScratchCarver sc{base};
    void* act_in = sc.take(e->state_elems * cs);
    void* act_out = sc.take(e->state_elems * cs);
    e->i1 = sc.take(e->i1_elems * cs);
    e->i2 = sc.take(e->i2_elems * cs);
    e->tw_x = sc.take(twx.size());
    e->tw_y = sc.take(twy.size());
    e->rho0_dev = static_cast<double*>(sc.take(sizeof(double)));
    e->err_dev = static_cast<int*>(sc.take(sizeof(int)));
    e->flag_dev = static_cast<int*>(sc.take(sizeof(int)));
    e->members_dev = static_cast<MemberInfo*>(sc.take(sizeof(MemberInfo)));
    if (sc.used > SHHD_NOALLOC_SCRATCH_BYTES)
        throw Failure(SHHD_EINVAL, "shhd_rhs_noalloc: this configuration needs " + std::to_string(sc.used) +
                                       " bytes of scratch but the static scratch holds " + std::to_string(SHHD_NOALLOC_SCRATCH_BYTES) +
                                       " bytes; use an engine (shhd_engine_create) for it");
    cudaStream_t s = e->stream;
    MemberInfo mi{};
    mi.key = static_cast<uint32_t>(e->cfg.member_offset);
    mi.active = 1;
    mi.step0 = 0;
    mi.noise_scale = 1.0;
    // the array keeps the previous call's contents: rewrite or clear everything read before written
    check_cuda(cudaMemcpyAsync(e->tw_x, twx.data(), twx.size(), cudaMemcpyHostToDevice, s), "twiddle upload");
    check_cuda(cudaMemcpyAsync(e->tw_y, twy.data(), twy.size(), cudaMemcpyHostToDevice, s), "twiddle upload");
    check_cuda(cudaMemcpyAsync(e->members_dev, &mi, sizeof(mi), cudaMemcpyHostToDevice, s), "member upload");
    check_cuda(cudaMemsetAsync(e->err_dev, 0, sizeof(int), s), "error word clear");
    check_cuda(cudaMemsetAsync(e->flag_dev, 0, sizeof(int), s), "flag clear");
    check_cuda(cudaMemsetAsync(act_out, 0, e->state_elems * cs, s), "rhs clear");

    // input checks of shhd_engine_set_state: nothing outside the active modes
    const int ref_hx = e->cfg.nx / 2 + 1;
    const double2* ref_in = reinterpret_cast<const double2*>(state_dev);
    {
        dim3 g((P.npy * ref_hx + kThreads - 1) / kThreads, P.nfields);
        check_inactive_kernel<<<g, kThreads, 0, s>>>(P, ref_hx, ref_in, e->flag_dev);
        check_cuda(cudaGetLastError(), "check_inactive launch");
    }
    int bad = 0;
    double rho00 = 0.0;
    check_cuda(cudaMemcpyAsync(&bad, e->flag_dev, sizeof(int), cudaMemcpyDeviceToHost, s), "flag read");
    check_cuda(cudaMemcpyAsync(&rho00, state_dev, sizeof(double), cudaMemcpyDeviceToHost, s), "density mode read");
    check_cuda(cudaStreamSynchronize(s), "input check sync");
    if (bad) throw Failure(SHHD_EINVAL, "state has a nonzero entry outside the active modes");
    // reference density of the incompressible terms (fcalculator_workspace.cc:41-66)
    double rho0 = rho00 / (static_cast<double>(e->cfg.nx) * e->cfg.ny);
    if (e->need_rho0 && rho0 == 0.0) throw Failure(SHHD_EINVAL, "reference density must be nonzero.");
    check_cuda(cudaMemcpyAsync(e->rho0_dev, &rho0, sizeof(double), cudaMemcpyHostToDevice, s), "rho0 upload");
    {
        dim3 g((P.hx * P.kyn + kThreads - 1) / kThreads, P.nfields);
        ref_to_active_kernel<T><<<g, kThreads, 0, s>>>(P, ref_hx, ref_in, static_cast<cplx<T>*>(act_in));
        check_cuda(cudaGetLastError(), "ref_to_active launch");
    }
    launch_col_inverse<T>(e, act_in);
    launch_row<T>(e);
    StageArgs<T> A = stage_args<T>(e, act_in, act_in, act_out, 0.0, 1.0, 0.0, 0, 0);
    A.det_mode = 1;
    launch_col_forward<T>(e, A);
    {
        dim3 g((P.npy * ref_hx + kThreads - 1) / kThreads, P.nfields);
        active_to_ref_kernel<T><<<g, kThreads, 0, s>>>(P, ref_hx, static_cast<const cplx<T>*>(act_out), reinterpret_cast<double2*>(rhs_dev));
        check_cuda(cudaGetLastError(), "active_to_ref launch");
    }
    int err = 0;
    check_cuda(cudaMemcpyAsync(&err, e->err_dev, sizeof(int), cudaMemcpyDeviceToHost, s), "error word read");
    check_cuda(cudaStreamSynchronize(s), "rhs sync");
    if (err & ERR_ZERO_DENSITY) throw Failure(SHHD_ENUMERIC, "compressible velocity encountered zero density.");
}

}  // namespace

extern "C" int shhd_rhs_noalloc(const shhd_config* cfg, const double* state_dev, double* rhs_dev, size_t n_doubles, void* stream) {
    return guarded([&] {
        if (!cfg) throw Failure(SHHD_EINVAL, "null configuration");
        if (cfg->batch != 1) throw Failure(SHHD_EINVAL, "shhd_rhs_noalloc evaluates one state: cfg->batch must be 1");
        // a host-side engine record only: its device pointers are set into the static scratch
        shhd_engine e;
        e.cfg = *cfg;
        validate_config(e.cfg);
        e.fp32 = cfg->precision == SHHD_FP32;
        e.csize = e.fp32 ? sizeof(float2) : sizeof(double2);
        build_plan(&e);
        if (n_doubles != ref_doubles(&e))
            throw Failure(SHHD_EINVAL, "state size mismatch: expected " + std::to_string(ref_doubles(&e)) + " doubles");
        check_cuda(cudaGetDevice(&e.device), "cudaGetDevice");
        e.stream = static_cast<cudaStream_t>(stream);
        // the call waits on its stream and reads results back: it cannot be recorded into a graph
        cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
        check_cuda(cudaStreamIsCapturing(e.stream, &capture), "cudaStreamIsCapturing");
        if (capture != cudaStreamCaptureStatusNone)
            throw Failure(SHHD_EINVAL, "shhd_rhs_noalloc is synchronous and cannot run on a stream that is being captured");
        check_device_buffer(state_dev, e.device, "state_dev");
        check_device_buffer(rhs_dev, e.device, "rhs_dev");
        unsigned char* base = noalloc_base();
        if (e.fp32) {
            set_smem_attrs<float>(&e);
            rhs_noalloc<float>(&e, state_dev, rhs_dev, base);
        } else {
            set_smem_attrs<double>(&e);
            rhs_noalloc<double>(&e, state_dev, rhs_dev, base);
        }
    });
}
