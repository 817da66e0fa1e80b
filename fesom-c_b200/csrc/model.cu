// C-ABI of the B200 FESOM-C time step: set-up of the device mesh (CSR
// gather lists in reference edge order), device state, the per-step launch
// sequence of oce_timestep case(3) (src/fv_main.F90:1983-2095) and its
// capture into one CUDA graph, forcing upload, state sync and diagnostics.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "closure.h"
#include "device_common.cuh"
#include "fesomc_gpu.h"
#include "forcing_dev.h"
#include "mlp.h"

namespace fesomc {
// kernels (k_*.cu), compiled once per precision
#define FESOMC_KERNEL_LAUNCHERS \
    void launch_ab3_elem(const Dev &, cudaStream_t); \
    void launch_ssh_node(const Dev &, int, cudaStream_t); \
    void launch_puls_elem(const Dev &, cudaStream_t); \
    void launch_el2nodes(const Dev &, const real *, const real *, real *, real *, cudaStream_t); \
    void launch_p1_edge(const Dev &, cudaStream_t); \
    void launch_p1_elem(const Dev &, cudaStream_t); \
    void launch_adv2d_edge(const Dev &, cudaStream_t); \
    void launch_u2d_elem(const Dev &, cudaStream_t); \
    void launch_rot_nodes(const Dev &, cudaStream_t); \
    void launch_zero_filt(const Dev &, cudaStream_t); \
    void launch_pressure_col(const Dev &, cudaStream_t); \
    void launch_bpg_elem(const Dev &, cudaStream_t); \
    void launch_velgrad3d(const Dev &, cudaStream_t); \
    void launch_adv3_edge(const Dev &, cudaStream_t); \
    void launch_velrhs(const Dev &, real, cudaStream_t); \
    void launch_bih(const Dev &, cudaStream_t); \
    void launch_filt2x(const Dev &, cudaStream_t); \
    void launch_filt2x_2d(const Dev &, cudaStream_t); \
    void launch_bih_2d(const Dev &, cudaStream_t); \
    void launch_bih_puls(const Dev &, cudaStream_t); \
    void launch_implvisc(const Dev &, cudaStream_t); \
    void launch_jac_swap(const Dev &, cudaStream_t); \
    void launch_je(const Dev &, cudaStream_t); \
    int config_d3end(const Dev &); \
    int config_vdiff(const Dev &); \
    int config_p1(const Dev &); \
    int config_columns(const Dev &); \
    void launch_ab2(const Dev &, cudaStream_t); \
    void launch_update3d(const Dev &, real, cudaStream_t); \
    void launch_wvel(const Dev &, cudaStream_t); \
    void launch_d3end(const Dev &, cudaStream_t); \
    void launch_av(const Dev &, cudaStream_t); \
    void launch_minmax(const Dev &, cudaStream_t); \
    void launch_aver_from_range(const Dev &, const double *, cudaStream_t); \
    void launch_atm(const Dev &, const AtmDev &, cudaStream_t); \
    void launch_upwind(const Dev &, cudaStream_t); \
    void launch_muscl_egrad(const Dev &, cudaStream_t); \
    void launch_muscl_ngrad(const Dev &, cudaStream_t); \
    void launch_muscl_edge(const Dev &, cudaStream_t); \
    void launch_miura(const Dev &, cudaStream_t); \
    void launch_muscl_h(const Dev &, cudaStream_t); \
    void launch_vdiff(const Dev &, cudaStream_t); \
    void launch_d3end_list(const Dev &, const int *, const unsigned long long *, cudaStream_t); \
    void launch_lc_features(const Dev &, const LcView &, cudaStream_t); \
    void launch_lc_apply(const Dev &, const LcView &, cudaStream_t); \
    void launch_lc_harvest(const Dev &, const LcView &, cudaStream_t); \
    void launch_lc_judge(const Dev &, const LcView &, cudaStream_t); \
    int energy_parts(); \
    int minmax_parts(int); \
    void tune_limits_baroclinic(int *); \
    void tune_limits_barotropic(int *); \
    void tune_limits_tracer(int *); \
    void tune_limits_mixing(int *); \
    void launch_energy(const Dev &, double *, double *, cudaStream_t);
namespace f64 {
FESOMC_KERNEL_LAUNCHERS
}  // namespace f64
namespace f32 {
FESOMC_KERNEL_LAUNCHERS
}  // namespace f32

int grid_for(long long n, int block) {
    long long g = (n + block - 1) / block;
    if (g < 1) g = 1;
    const long long cap = 148LL * 32;
    return (int)(g < cap ? g : cap);
}

// Harmonics_tf_period (fv_var.F90:171-172), hours
static const double kHarmPeriod[12] = {12.4200, 12.00, 12.6584, 11.9673, 23.9344, 25.8194,
                                       24.0659, 26.8684, 327.85, 661.31, 4383.05, 6.2103};
static const double kPi = 3.14159265358979;
}  // namespace fesomc

using namespace fesomc;
using namespace fesomc::f64;

// a halo plan (fesomc_gpu_halo_plan): nodes and elements of one model
struct fesomc_halo {
    int n_nodes = 0, n_elems = 0;
    int *d_nodes = nullptr, *d_elems = nullptr;   // device order
    long long count = 0;                          // doubles per buffer
    double *d_range = nullptr;                    // min / max scratch
};

struct fesomc_model {
    Dev d{};                    // FP64 view: 2D sub-cycle (always) and, in the FP64 form, everything
    fesomc::f32::Dev d32{};     // FP32 form: level fields, geometry and 3D arithmetic in FP32
    bool fp32 = false;
    std::vector<float> h_f32;   // host staging for FP32 level fields
    fesomc_params p{};
    cudaStream_t stream = nullptr;
    std::vector<void *> allocs;
    // host copies needed per step
    std::vector<double> ampt, fazt;
    double amp_factor[12], phy_factor[12];
    // pinned staging for per-step uploads (double buffered)
    double *h_stage[2] = {nullptr, nullptr};
    cudaEvent_t stage_ev[2] = {nullptr, nullptr};
    int stage_i = 0;
    size_t stage_len = 0;
    double *h_runoff = nullptr;  // host copy of current runoff
    // open-boundary table of the next step, evaluated while the GPU runs the
    // current one (valid for pre_time_jd and the current harmonics)
    std::vector<double> h_pre;
    double pre_time_jd = 0.0;
    bool pre_valid = false;
    bool runoff_dirty = false;
    // asynchronous snapshots (fesomc_gpu_snapshot_begin / _end)
    struct Snap {
        double *dst;                  // caller's array (FP64)
        void *dev_copy;
        float *pinned32;              // FP32 fields: pinned staging, converted in _end
        size_t count;
    };
    std::vector<Snap> snaps;          // fields of the snapshot in flight
    std::vector<std::pair<void *, float *>> snap_bufs;  // (device copy, FP32 staging) per field slot
    std::vector<size_t> snap_bytes;
    std::vector<std::pair<void *, size_t>> registered;  // caller arrays page-locked for direct copies
    fesomc_state *snap_state = nullptr;
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t snap_taken = nullptr, snap_done = nullptr;
    bool snap_pending = false;
    double snap_time_jd = 0.0;
    int snap_lfirst = 0;
    // forcing on the device (fesomc_gpu_set_device_forcing)
    bool dev_forcing = false;
    int river_ramp = 0;
    bool have_jer = false;                  // key_atm with jer_const = 0: Rj, aj, bj given
    double *d_clock = nullptr, *d_ampt = nullptr, *d_fazt = nullptr, *d_harm = nullptr, *d_runoff_base = nullptr;
    const double2 *d_coord = nullptr;       // node (lon, lat) for the tidal potential
    // diagnostics
    double *d_epart = nullptr, *d_eout = nullptr;
    unsigned int *h_status = nullptr;
    int *h_notconv = nullptr;
    unsigned int status_acc = 0;
    int notconv_acc = 0;
    // time
    double time_jd = 0.0;
    int lfirst = 1;
    // learned closure (fesomc_closure_attach / _harvest): the network in use,
    // its per-column buffers, and what the coming step does with it
    fesomc::LcNet *lc = nullptr;
    fesomc::LcView lcv{};
    float *lc_bufA = nullptr, *lc_bufB = nullptr;
    bool lc_on = false;               // the network stands in for d3_end
    bool lc_bf16 = false;             // inference on the tensor cores (BF16) instead of FP32
    bool lc_judge_now = false;        // this step: plain closure on every column, compared
    bool lc_harvest_now = false;      // this step: plain closure, columns harvested
    int lc_judge_every = 0;
    long long lc_steps = 0, lc_judges = 0;
    void *lc_owner = nullptr;         // fesomc_closure the per-column buffers were made for
    // packed members (fesomc_gpu_init_packed): node and element ranges of
    // each member in the reference numbering of the packed mesh
    int n_members = 1;
    std::vector<int> member_node_off, member_elem_off;
    std::vector<double> member_scale_area;
    // storage order (fesomc_params.sfc_order): device index -> reference
    // index of nodes and elements, used by every transfer of a field
    bool perm = false;
    const int *d_nd_ref = nullptr, *d_el_ref = nullptr;
    void *d_perm_buf = nullptr;       // staging of one field in reference order
    size_t perm_buf_bytes = 0;
    // sbc_do on the device (fesomc_gpu_set_atm_fields): the atmospheric
    // fields' time-interpolation coefficients (device order) and the stress
    // per node
    bool dev_atm = false;
    double *d_atm_a = nullptr, *d_atm_b = nullptr, *d_tau_node = nullptr;
    int atm_net_flux = 0;
    double atm_prec_coef = 1.0;
    // tracer range given by the host (fesomc_gpu_set_tracer_range): tmin,
    // tmax, smin, smax on the device, replacing the step's own min / max
    bool ext_range = false;
    double *d_ext_range = nullptr;
    // graph
    cudaGraphExec_t graph = nullptr;
    bool use_graph = true;
    long long launches = 0;
    int launches_per_step = 0;
    // optional per-kernel profiling (events around every launch group)
    struct Prof {
        bool on = false;
        std::vector<std::string> names;
        std::vector<double> bytes, ms;
        std::vector<long long> count;
        std::vector<cudaEvent_t> ev;      // pool, 2 per record
        std::vector<int> rec_kernel;      // kernel index of each record
        size_t used = 0;
    } prof;
};

namespace {

#define CK(x)                                                                           \
    do {                                                                                \
        cudaError_t e_ = (x);                                                           \
        if (e_ != cudaSuccess) {                                                        \
            std::fprintf(stderr, "fesomc: CUDA error %s at %s:%d\n", cudaGetErrorString(e_), \
                         __FILE__, __LINE__);                                           \
            return FESOMC_ECUDA;                                                        \
        }                                                                               \
    } while (0)

template <typename T>
int dalloc(fesomc_model *m, T **p, size_t n) {
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, (n ? n : 1) * sizeof(T));
    if (e != cudaSuccess) return FESOMC_ENOMEM;
    // the zero fill runs on the legacy default stream, which the model's
    // non-blocking streams do not wait for: let it land before anything
    // is enqueued on them (an upload into a buffer allocated just before
    // could otherwise be overwritten by the fill)
    cudaMemset(q, 0, (n ? n : 1) * sizeof(T));
    if (cudaDeviceSynchronize() != cudaSuccess) {
        cudaFree(q);
        return FESOMC_ECUDA;
    }
    m->allocs.push_back(q);
    *p = static_cast<T *>(q);
    return FESOMC_OK;
}

template <typename T>
int upload(fesomc_model *m, const T **dst, const std::vector<T> &src) {
    T *q = nullptr;
    int rc = dalloc(m, &q, src.size());
    if (rc) return rc;
    if (!src.empty()) CK(cudaMemcpy(q, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice));
    *dst = q;
    return FESOMC_OK;
}

// Storage order: fields live on the device in the order of the model's
// nodes / elements, which with fesomc_params.sfc_order is a Hilbert-curve
// order of the mesh; callers always see the reference order.  A field of an
// entity kind holds 'lev' consecutive values per entity.
template <typename T>
__global__ void k_perm_gather(const T *ref, T *dev, const int *ref_of, long long n_ent, int lev) {
    const long long total = n_ent * lev;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const long long e = i / lev, k = i % lev;
        dev[i] = ref[(size_t)ref_of[e] * lev + k];
    }
}
template <typename T>
__global__ void k_perm_scatter(const T *dev, T *ref, const int *ref_of, long long n_ent, int lev) {
    const long long total = n_ent * lev;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const long long e = i / lev, k = i % lev;
        ref[(size_t)ref_of[e] * lev + k] = dev[i];
    }
}

// halo exchange of a decomposed mesh (fesomc_gpu_halo_*)
template <typename T>
__global__ void k_halo_gather(const T *src, int width, const int *idx, int n, double *dst) {
    const long long total = (long long)n * width;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / width, c = i - r * width;
        dst[i] = (double)src[(size_t)idx[r] * width + c];
    }
}
template <typename T>
__global__ void k_halo_scatter(T *dst, int width, const int *idx, int n, const double *src) {
    const long long total = (long long)n * width;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / width, c = i - r * width;
        dst[(size_t)idx[r] * width + c] = (T)src[i];
    }
}
// min / max of two fields of width w over the listed entities: one block
template <typename T>
__global__ void k_halo_range(const T *a, const T *b, int w, const int *idx, int n, double *out) {
    __shared__ double s[4][256];
    double amin = (double)a[(size_t)idx[0] * w], amax = amin, bmin = (double)b[(size_t)idx[0] * w], bmax = bmin;
    for (long long i = threadIdx.x; i < (long long)n * w; i += blockDim.x) {
        const size_t g = (size_t)idx[i / w] * w + (size_t)(i % w);
        const double x = (double)a[g], y = (double)b[g];
        amin = fmin(amin, x); amax = fmax(amax, x);
        bmin = fmin(bmin, y); bmax = fmax(bmax, y);
    }
    s[0][threadIdx.x] = amin; s[1][threadIdx.x] = amax; s[2][threadIdx.x] = bmin; s[3][threadIdx.x] = bmax;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            s[0][threadIdx.x] = fmin(s[0][threadIdx.x], s[0][threadIdx.x + o]);
            s[1][threadIdx.x] = fmax(s[1][threadIdx.x], s[1][threadIdx.x + o]);
            s[2][threadIdx.x] = fmin(s[2][threadIdx.x], s[2][threadIdx.x + o]);
            s[3][threadIdx.x] = fmax(s[3][threadIdx.x], s[3][threadIdx.x + o]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) { out[0] = s[0][0]; out[1] = s[1][0]; out[2] = s[2][0]; out[3] = s[3][0]; }
}

enum { ENT_NODE = 0, ENT_ELEM = 1 };

// the permutation of an entity kind and the values per entity of a field
inline const int *perm_of(const fesomc_model *m, int ent) { return ent == ENT_NODE ? m->d_nd_ref : m->d_el_ref; }
inline long long ents(const fesomc_model *m, int ent) { return ent == ENT_NODE ? m->d.N : m->d.E; }

int perm_buf(fesomc_model *m, size_t bytes) {
    if (m->perm_buf_bytes >= bytes) return FESOMC_OK;
    unsigned char *q = nullptr;
    int rc = dalloc(m, &q, bytes);
    if (rc) return rc;
    m->d_perm_buf = q;
    m->perm_buf_bytes = bytes;
    return FESOMC_OK;
}

// device field (device order) -> buffer in reference order, on stream s
template <typename T>
void unpermute_to(const fesomc_model *m, int ent, const T *dev, T *ref, size_t count, cudaStream_t s) {
    const long long n = ents(m, ent);
    const int lev = (int)(count / n);
    k_perm_scatter<<<grid_for(count, 256), 256, 0, s>>>(dev, ref, perm_of(m, ent), n, lev);
}
template <typename T>
void permute_from(const fesomc_model *m, int ent, const T *ref, T *dev, size_t count, cudaStream_t s) {
    const long long n = ents(m, ent);
    const int lev = (int)(count / n);
    k_perm_gather<<<grid_for(count, 256), 256, 0, s>>>(ref, dev, perm_of(m, ent), n, lev);
}

// field table for state sync: name of the fesomc_state member, device
// pointer, count, group, whether the device copy is FP32 (level fields and
// 2D momentum of the FP32 form), and the entity kind it is stored per
struct FieldRef {
    double *fesomc_state::*host;
    void *dev;
    size_t count;
    uint32_t group;
    bool f32;
    int ent;
};

std::vector<FieldRef> field_table(fesomc_model *m) {
    Dev &d = m->d;
    fesomc::f32::Dev &q = m->d32;
    const bool f = m->fp32;
    const size_t N = d.N, E = d.E, L = d.L, NS = d.NS;
#define LEV(name) (f ? (void *)q.name : (void *)d.name)
    return {
        {&fesomc_state::eta_n, d.eta_n, N, FESOMC_F_ETA, false, ENT_NODE},
        {&fesomc_state::eta_n_1, d.eta_n_1, N, FESOMC_F_ETA, false, ENT_NODE},
        {&fesomc_state::eta_n_2, d.eta_n_2, N, FESOMC_F_ETA, false, ENT_NODE},
        {&fesomc_state::etaAB, d.etaAB, N, FESOMC_F_ETA, false, ENT_NODE},
        {&fesomc_state::ssh_gp, d.ssh_gp, N, FESOMC_F_ETA, false, ENT_NODE},
        {&fesomc_state::U_n_2D, LEV(U_n_2D), 2 * E, FESOMC_F_UV2D, f, ENT_ELEM},
        {&fesomc_state::U_n_1, LEV(U_n_1), 2 * E, FESOMC_F_UV2D, f, ENT_ELEM},
        {&fesomc_state::U_n_2, LEV(U_n_2), 2 * E, FESOMC_F_UV2D, f, ENT_ELEM},
        {&fesomc_state::U_filt_2D, LEV(U_filt_2D), E, FESOMC_F_UV2D, f, ENT_ELEM},
        {&fesomc_state::V_filt_2D, LEV(V_filt_2D), E, FESOMC_F_UV2D, f, ENT_ELEM},
        {&fesomc_state::U_n, LEV(U_n), L * E, FESOMC_F_UV3D, f, ENT_ELEM},
        {&fesomc_state::V_n, LEV(V_n), L * E, FESOMC_F_UV3D, f, ENT_ELEM},
        {&fesomc_state::U_rhsAB, LEV(U_rhsAB), L * E, FESOMC_F_UV3D, f, ENT_ELEM},
        {&fesomc_state::V_rhsAB, LEV(V_rhsAB), L * E, FESOMC_F_UV3D, f, ENT_ELEM},
        {&fesomc_state::U_n_filt, LEV(U_n_filt), L * E, FESOMC_F_UV3D, f, ENT_ELEM},
        {&fesomc_state::V_n_filt, LEV(V_n_filt), L * E, FESOMC_F_UV3D, f, ENT_ELEM},
        {&fesomc_state::TF, LEV(TF), L * N, FESOMC_F_TS, f, ENT_NODE},
        {&fesomc_state::SF, LEV(SF), L * N, FESOMC_F_TS, f, ENT_NODE},
        {&fesomc_state::T_old, LEV(T_old), L * N, FESOMC_F_TS, f, ENT_NODE},
        {&fesomc_state::S_old, LEV(S_old), L * N, FESOMC_F_TS, f, ENT_NODE},
        {&fesomc_state::Tclim, LEV(Tclim), L * N, FESOMC_F_CLIM, f, ENT_NODE},
        {&fesomc_state::Sclim, LEV(Sclim), L * N, FESOMC_F_CLIM, f, ENT_NODE},
        {&fesomc_state::bt, LEV(bt), NS * N, FESOMC_F_MIX, f, ENT_NODE},
        {&fesomc_state::snu, LEV(snu), NS * N, FESOMC_F_MIX, f, ENT_NODE},
        {&fesomc_state::Kv, LEV(Kv), NS * N, FESOMC_F_MIX, f, ENT_NODE},
        {&fesomc_state::Ri, LEV(Ri), NS * N, FESOMC_F_MIX, f, ENT_NODE},
        {&fesomc_state::tke_dissip, LEV(tke_dissip), NS * N, FESOMC_F_MIX, f, ENT_NODE},
        {&fesomc_state::Av, LEV(Av), NS * E, FESOMC_F_MIX, f, ENT_ELEM},
        {&fesomc_state::Wvel, LEV(Wvel), NS * N, FESOMC_F_WVEL, f, ENT_NODE},
        {&fesomc_state::mask_wd, LEV(mask_wd), E, FESOMC_F_MASK, f, ENT_ELEM},
        {&fesomc_state::mask_wd_node, LEV(mask_wd_node), N, FESOMC_F_MASK, f, ENT_NODE},
        {&fesomc_state::rho_c, LEV(rho_c), L * N, FESOMC_F_DIAG, f, ENT_NODE},
        {&fesomc_state::hpressure, LEV(hpressure), NS * N, FESOMC_F_DIAG, f, ENT_NODE},
        {&fesomc_state::Bar_pr_2D, LEV(Bar_pr_2D), 2 * E, FESOMC_F_DIAG, f, ENT_ELEM},
    };
#undef LEV
}

// host double <-> device field (converting for FP32 level fields, and
// between the reference and the storage order)
int field_to_host(fesomc_model *m, const FieldRef &f, double *h) {
    const size_t bytes = f.count * (f.f32 ? sizeof(float) : sizeof(double));
    const void *src = f.dev;
    if (m->perm) {
        int rc = perm_buf(m, bytes);
        if (rc) return rc;
        if (f.f32) unpermute_to(m, f.ent, (const float *)f.dev, (float *)m->d_perm_buf, f.count, m->stream);
        else unpermute_to(m, f.ent, (const double *)f.dev, (double *)m->d_perm_buf, f.count, m->stream);
        src = m->d_perm_buf;
    }
    // the model's stream is non-blocking: copy on it, then wait for it
    if (!f.f32) {
        CK(cudaMemcpyAsync(h, src, bytes, cudaMemcpyDeviceToHost, m->stream));
        CK(cudaStreamSynchronize(m->stream));
        return FESOMC_OK;
    }
    m->h_f32.resize(f.count);
    CK(cudaMemcpyAsync(m->h_f32.data(), src, bytes, cudaMemcpyDeviceToHost, m->stream));
    CK(cudaStreamSynchronize(m->stream));
    for (size_t i = 0; i < f.count; ++i) h[i] = (double)m->h_f32[i];
    return FESOMC_OK;
}
int field_from_host(fesomc_model *m, void *dev, bool f32, size_t count, const double *h, int ent) {
    const size_t bytes = count * (f32 ? sizeof(float) : sizeof(double));
    void *dst = dev;
    if (m->perm) {
        int rc = perm_buf(m, bytes);
        if (rc) return rc;
        dst = m->d_perm_buf;
    }
    // on the model's (non-blocking) stream, so that the permutation below
    // reads the staging buffer after the copy into it has landed
    if (!f32) {
        CK(cudaMemcpyAsync(dst, h, bytes, cudaMemcpyHostToDevice, m->stream));
    } else {
        m->h_f32.resize(count);
        for (size_t i = 0; i < count; ++i) m->h_f32[i] = (float)h[i];
        CK(cudaMemcpyAsync(dst, m->h_f32.data(), bytes, cudaMemcpyHostToDevice, m->stream));
    }
    if (m->perm) {
        if (f32) permute_from(m, ent, (const float *)m->d_perm_buf, (float *)dev, count, m->stream);
        else permute_from(m, ent, (const double *)m->d_perm_buf, (double *)dev, count, m->stream);
    }
    CK(cudaStreamSynchronize(m->stream));
    return FESOMC_OK;
}

// Hilbert-curve index of (x, y) on an n x n grid, n a power of two
uint64_t hilbert_index(uint32_t n, uint32_t x, uint32_t y) {
    uint64_t d = 0;
    for (uint32_t s = n / 2; s > 0; s /= 2) {
        const uint32_t rx = (x & s) > 0, ry = (y & s) > 0;
        d += (uint64_t)s * s * ((3 * rx) ^ ry);
        if (ry == 0) {
            if (rx == 1) { x = n - 1 - x; y = n - 1 - y; }
            std::swap(x, y);
        }
    }
    return d;
}

// Storage order of nodes, elements and edges: identity, or (sfc_order) the
// order of a Hilbert curve through the node positions, element centroids and
// edge midpoints, internal and boundary edges each kept in their own range
// (the kernels tell them apart by index).  *_ref maps a device index to the
// reference one, *_dev the reverse.
//
// Packed members (node_member / elem_member non-empty, reference numbering):
// each member's nodes and elements stay in its own contiguous range, the
// curve ordering them within it, and edges are ordered by their member first.
void storage_order(const fesomc_mesh *msh, bool sfc, const std::vector<int> &node_member,
                   const std::vector<int> &elem_member, std::vector<int> &nd_ref, std::vector<int> &el_ref,
                   std::vector<int> &ed_ref) {
    const int N = msh->nod2D, E = msh->elem2D, Ed = msh->edge2D, Ed_in = msh->edge2D_in;
    nd_ref.resize(N); el_ref.resize(E); ed_ref.resize(Ed);
    for (int i = 0; i < N; ++i) nd_ref[i] = i;
    for (int i = 0; i < E; ++i) el_ref[i] = i;
    for (int i = 0; i < Ed; ++i) ed_ref[i] = i;
    if (!sfc || !msh->coord_nod2D) return;
    const double *c = msh->coord_nod2D;
    double x0 = c[0], x1 = c[0], y0 = c[1], y1 = c[1];
    for (int i = 0; i < N; ++i) {
        x0 = std::min(x0, c[2 * i]); x1 = std::max(x1, c[2 * i]);
        y0 = std::min(y0, c[2 * i + 1]); y1 = std::max(y1, c[2 * i + 1]);
    }
    const uint32_t G = 1u << 16;
    const double sx = (x1 > x0) ? (G - 1) / (x1 - x0) : 0.0, sy = (y1 > y0) ? (G - 1) / (y1 - y0) : 0.0;
    auto key = [&](double x, double y) {
        return hilbert_index(G, (uint32_t)((x - x0) * sx), (uint32_t)((y - y0) * sy));
    };
    const bool packed = !node_member.empty();
    auto mkey = [&](int member) { return packed ? (uint64_t)member << 40 : (uint64_t)0; };
    auto order = [](std::vector<int> &idx, int lo, int hi, const std::vector<uint64_t> &k) {
        std::sort(idx.begin() + lo, idx.begin() + hi, [&](int a, int b) { return k[a] != k[b] ? k[a] < k[b] : a < b; });
    };
    std::vector<uint64_t> kn(N), ke(E), kd(Ed);
    for (int i = 0; i < N; ++i) kn[i] = mkey(packed ? node_member[i] : 0) | key(c[2 * i], c[2 * i + 1]);
    for (int e = 0; e < E; ++e) {
        const int32_t *q = msh->elem2D_nodes + 4 * e;
        const int q1 = (q[0] == q[3]) ? 3 : 4;
        double x = 0.0, y = 0.0;
        for (int k = 0; k < q1; ++k) { x += c[2 * (q[k] - 1)]; y += c[2 * (q[k] - 1) + 1]; }
        ke[e] = mkey(packed ? elem_member[e] : 0) | key(x / q1, y / q1);
    }
    for (int ed = 0; ed < Ed; ++ed) {
        const int a = msh->edge_nodes[2 * ed] - 1, b = msh->edge_nodes[2 * ed + 1] - 1;
        kd[ed] = mkey(packed ? node_member[a] : 0) | key(0.5 * (c[2 * a] + c[2 * b]), 0.5 * (c[2 * a + 1] + c[2 * b + 1]));
    }
    order(nd_ref, 0, N, kn);
    order(el_ref, 0, E, ke);
    order(ed_ref, 0, Ed_in, kd);
    order(ed_ref, Ed_in, Ed, kd);
}

std::vector<int> inverse(const std::vector<int> &ref) {
    std::vector<int> dev(ref.size());
    for (size_t i = 0; i < ref.size(); ++i) dev[ref[i]] = (int)i;
    return dev;
}

int build_mesh(fesomc_model *m, const fesomc_mesh *msh) {
    Dev &d = m->d;
    const int N = msh->nod2D, E = msh->elem2D, Ed = msh->edge2D, Ed_in = msh->edge2D_in, NS = msh->nsigma;
    const int L = NS - 1;
    d.N = N; d.E = E; d.Ed = Ed; d.Ed_in = Ed_in; d.L = L; d.NS = NS;
    d.nobn = msh->nobn; d.n_rivers = msh->n_rivers;
    std::vector<double> sig(msh->sigma, msh->sigma + NS), dsig(L);
    for (int k = 0; k < L; ++k) dsig[k] = sig[k] - sig[k + 1];
    int rc;
    if ((rc = upload(m, &d.sig, sig)) || (rc = upload(m, &d.dsig, dsig))) return rc;
    // connectivity checks, in reference numbering
    for (int e = 0; e < E; ++e)
        for (int k = 0; k < 4; ++k) {
            const int32_t q = msh->elem2D_nodes[4 * e + k], g = msh->elem_edges[4 * e + k];
            if (q < 1 || q > N) return FESOMC_EINVAL;
            if (k < ((msh->elem2D_nodes[4 * e] == msh->elem2D_nodes[4 * e + 3]) ? 3 : 4) && (g < 1 || g > Ed))
                return FESOMC_EINVAL;
        }
    for (int ed = 0; ed < Ed; ++ed) {
        const int n1 = msh->edge_nodes[2 * ed], n2 = msh->edge_nodes[2 * ed + 1];
        if (n1 < 1 || n1 > N || n2 < 1 || n2 > N) return FESOMC_EINVAL;
        const int t1 = msh->edge_tri[2 * ed], t2 = msh->edge_tri[2 * ed + 1];
        if (t1 < 1 || t1 > E) return FESOMC_EINVAL;
        if ((ed < Ed_in) != (t2 > 0)) return FESOMC_EINVAL;
    }
    // packed members: the member of every node and element (reference numbering)
    std::vector<int> nmem, emem;
    if (m->n_members > 1) {
        nmem.resize(N);
        emem.resize(E);
        for (int k = 0; k < m->n_members; ++k) {
            for (int i = m->member_node_off[k]; i < m->member_node_off[k + 1]; ++i) nmem[i] = k;
            for (int i = m->member_elem_off[k]; i < m->member_elem_off[k + 1]; ++i) emem[i] = k;
        }
    }
    std::vector<int> nd_ref, el_ref, ed_ref;
    storage_order(msh, m->p.sfc_order != 0, nmem, emem, nd_ref, el_ref, ed_ref);
    const std::vector<int> nd_dev = inverse(nd_ref), el_dev = inverse(el_ref), ed_dev = inverse(ed_ref);
    m->perm = m->p.sfc_order != 0;
    if (m->perm && ((rc = upload(m, &m->d_nd_ref, nd_ref)) || (rc = upload(m, &m->d_el_ref, el_ref)))) return rc;
    auto ndv = [&](int ref1) { return nd_dev[ref1 - 1]; };        // 1-based reference node -> device
    auto elv = [&](int ref1) { return ref1 > 0 ? el_dev[ref1 - 1] : -1; };
    // an edge list entry: device edge and side, sorted by the reference edge number
    auto edge_codes = [&](const int *refcodes, int n, int *out) {
        int tmp[4];
        for (int t = 0; t < n; ++t) tmp[t] = refcodes[t];
        for (int a = 1; a < n; ++a)
            for (int b2 = a; b2 > 0 && tmp[b2 - 1] > tmp[b2]; --b2) std::swap(tmp[b2 - 1], tmp[b2]);
        for (int t = 0; t < 4; ++t) out[t] = t < n ? ((ed_dev[tmp[t] >> 1] << 1) | (tmp[t] & 1)) : -1;
    };
    std::vector<int4> en(E), nb(E), ee(E), iel(E), sel(E);
    std::vector<double4> wcv(E), gsx(E), gsy(E), gvx(E), gvy(E);
    std::vector<double> eacc(E), bpf(E);
    for (int ei = 0; ei < E; ++ei) {
        const int e = el_ref[ei];
        const int32_t *q = msh->elem2D_nodes + 4 * e;
        en[ei] = make_int4(ndv(q[0]), ndv(q[1]), ndv(q[2]), ndv(q[3]));
        const int32_t *b = msh->elem_neighbors + 4 * e;
        nb[ei] = make_int4(elv(b[0]), elv(b[1]), elv(b[2]), elv(b[3]));
        const int32_t *g = msh->elem_edges + 4 * e;
        ee[ei] = make_int4(g[0] > 0 ? ed_dev[g[0] - 1] : -1, g[1] > 0 ? ed_dev[g[1] - 1] : -1,
                           g[2] > 0 ? ed_dev[g[2] - 1] : -1, g[3] > 0 ? ed_dev[g[3] - 1] : -1);
        const double *w = msh->w_cv + 4 * e;
        wcv[ei] = make_double4(w[0], w[1], w[2], w[3]);
        const double *sg = msh->gradient_sca + 8 * e;
        gsx[ei] = make_double4(sg[0], sg[1], sg[2], sg[3]);
        gsy[ei] = make_double4(sg[4], sg[5], sg[6], sg[7]);
        const double *v = msh->gradient_vec + 8 * e;
        gvx[ei] = make_double4(v[0], v[1], v[2], v[3]);
        gvy[ei] = make_double4(v[4], v[5], v[6], v[7]);
        double acc = 0.0;
        for (int k = 0; k < 4; ++k) acc = acc + w[k] * msh->ac[q[k] - 1];
        eacc[ei] = acc;
        bpf[ei] = std::pow(acc, m->p.Bp_bz) * 1.0;
        // internal edges of this element, in reference edge order, with the
        // side; and all its edges (boundary ones too)
        const int q1 = (q[0] == q[3]) ? 3 : 4;
        int list[4], nl = 0, all[4], na = 0;
        for (int j = 0; j < q1; ++j) {
            const int edg = g[j];
            const int code = ((edg - 1) << 1) | ((msh->edge_tri[2 * (edg - 1)] == e + 1) ? 0 : 1);
            bool dup = false;
            for (int t = 0; t < na; ++t) dup |= ((all[t] >> 1) == edg - 1);
            if (dup) continue;
            all[na++] = code;
            if (edg <= Ed_in) list[nl++] = code;
        }
        int o1[4], o2[4];
        edge_codes(list, nl, o1);
        edge_codes(all, na, o2);
        iel[ei] = make_int4(o1[0], o1[1], o1[2], o1[3]);
        sel[ei] = make_int4(o2[0], o2[1], o2[2], o2[3]);
    }
    std::vector<int2> edn(Ed), edt(Ed), eud(Ed);
    std::vector<double2> exy(Ed);
    std::vector<double4> ecr(Ed);
    std::vector<int> ecount(N + 1, 0), bcount(N + 1, 0);
    for (int di = 0; di < Ed; ++di) {
        const int ed = ed_ref[di];
        const int n1 = msh->edge_nodes[2 * ed], n2 = msh->edge_nodes[2 * ed + 1];
        edn[di] = make_int2(ndv(n1), ndv(n2));
        edt[di] = make_int2(elv(msh->edge_tri[2 * ed]), elv(msh->edge_tri[2 * ed + 1]));
        if (msh->edge_up_dn_tri) {
            const int u = msh->edge_up_dn_tri[2 * ed], w = msh->edge_up_dn_tri[2 * ed + 1];
            eud[di] = make_int2(elv(u), elv(w));
        } else {
            eud[di] = make_int2(-1, -1);
        }
        exy[di] = make_double2(msh->edge_dxdy[2 * ed], msh->edge_dxdy[2 * ed + 1]);
        const double *cc = msh->edge_cross_dxdy + 4 * ed;
        ecr[di] = make_double4(cc[0], cc[1], cc[2], cc[3]);
        ecount[edn[di].x + 1]++; ecount[edn[di].y + 1]++;
        if (ed >= Ed_in) { bcount[edn[di].x + 1]++; bcount[edn[di].y + 1]++; }
    }
    // CSR node -> edges, each list in reference edge order
    std::vector<int> eptr(N + 1, 0), bptr(N + 1, 0);
    for (int n = 0; n < N; ++n) { eptr[n + 1] = eptr[n] + ecount[n + 1]; bptr[n + 1] = bptr[n] + bcount[n + 1]; }
    std::vector<int> eidx(eptr[N]), bidx(bptr[N]), efill(eptr.begin(), eptr.end() - 1), bfill(bptr.begin(), bptr.end() - 1);
    for (int ed = 0; ed < Ed; ++ed) {
        const int di = ed_dev[ed];
        eidx[efill[edn[di].x]++] = (di << 1) | 0;
        eidx[efill[edn[di].y]++] = (di << 1) | 1;
        if (ed >= Ed_in) {
            bidx[bfill[edn[di].x]++] = (di << 1) | 0;
            bidx[bfill[edn[di].y]++] = (di << 1) | 1;
        }
    }
    // CSR node -> elements (nod_in_elem2D order) and the summed area
    std::vector<int> nptr(N + 1, 0), nidx;
    std::vector<double> tvol(N);
    for (int ni = 0; ni < N; ++ni) {
        const int n = nd_ref[ni];
        const int num = msh->nod_in_elem2D_num[n];
        double sum = 0.0;
        for (int k = 0; k < num; ++k) {
            const int el = msh->nod_in_elem2D[(size_t)msh->nod_in_elem2D_max * n + k];
            if (el < 1 || el > E) return FESOMC_EINVAL;
            nidx.push_back(el_dev[el - 1]);
            sum = sum + msh->elem_area[el - 1];
        }
        nptr[ni + 1] = (int)nidx.size();
        tvol[ni] = sum;
    }
    // rivers and open boundary
    std::vector<int> rcount(N + 1, 0);
    for (int i = 0; i < msh->n_rivers; ++i) {
        const int nd = msh->nod_rivers[i];
        if (nd < 1 || nd > N) return FESOMC_EINVAL;
        rcount[ndv(nd) + 1]++;
    }
    std::vector<int> rptr(N + 1, 0);
    for (int n = 0; n < N; ++n) rptr[n + 1] = rptr[n] + rcount[n + 1];
    std::vector<int> ridx(rptr[N]), rfill(rptr.begin(), rptr.end() - 1);
    for (int i = 0; i < msh->n_rivers; ++i) ridx[rfill[ndv(msh->nod_rivers[i])]++] = i;
    std::vector<int> obn(N, -1);
    for (int i = 0; i < msh->nobn; ++i) {
        const int nd = msh->in_obn[i];
        if (nd < 1 || nd > N) return FESOMC_EINVAL;
        obn[ndv(nd)] = i;
    }
    // per-node and per-element mesh arrays in storage order
    auto gather_n = [&](const double *src) { std::vector<double> v(N); for (int i = 0; i < N; ++i) v[i] = src[nd_ref[i]]; return v; };
    auto gather_e = [&](const double *src) { std::vector<double> v(E); for (int i = 0; i < E; ++i) v[i] = src[el_ref[i]]; return v; };
    std::vector<int> idx(N);
    for (int i = 0; i < N; ++i) idx[i] = msh->index_nod2D[nd_ref[i]];
    std::vector<double> dep = gather_n(msh->depth), area = gather_n(msh->area), ac = gather_n(msh->ac);
    std::vector<double> atp1 = gather_n(msh->a_tp), atp2 = gather_n(msh->a_tp + N);
    std::vector<double> ea = gather_e(msh->elem_area), ec = gather_e(msh->elem_cos), cor = gather_e(msh->coriolis);
    if ((rc = upload(m, &d.elem_nodes, en)) || (rc = upload(m, &d.elem_nb, nb)) || (rc = upload(m, &d.elem_edges, ee)) ||
        (rc = upload(m, &d.elem_iedges, iel)) || (rc = upload(m, &d.elem_sedges, sel)) ||
        (rc = upload(m, &d.edge_nodes, edn)) ||
        (rc = upload(m, &d.edge_tri, edt)) || (rc = upload(m, &d.edge_updn, eud)) ||
        (rc = upload(m, &d.node_eptr, eptr)) || (rc = upload(m, &d.node_eidx, eidx)) ||
        (rc = upload(m, &d.node_nptr, nptr)) || (rc = upload(m, &d.node_nidx, nidx)) ||
        (rc = upload(m, &d.node_bptr, bptr)) || (rc = upload(m, &d.node_bidx, bidx)) ||
        (rc = upload(m, &d.node_rptr, rptr)) || (rc = upload(m, &d.node_ridx, ridx)) ||
        (rc = upload(m, &d.obn_of_node, obn)) || (rc = upload(m, &d.index_nod2D, idx)) ||
        (rc = upload(m, &d.w_cv, wcv)) || (rc = upload(m, &d.gs_x, gsx)) || (rc = upload(m, &d.gs_y, gsy)) ||
        (rc = upload(m, &d.gv_x, gvx)) || (rc = upload(m, &d.gv_y, gvy)) || (rc = upload(m, &d.elem_area, ea)) ||
        (rc = upload(m, &d.elem_cos, ec)) || (rc = upload(m, &d.coriolis, cor)) || (rc = upload(m, &d.area, area)) ||
        (rc = upload(m, &d.depth, dep)) || (rc = upload(m, &d.ac, ac)) || (rc = upload(m, &d.atp1, atp1)) ||
        (rc = upload(m, &d.atp2, atp2)) || (rc = upload(m, &d.elem_acc, eacc)) ||
        (rc = upload(m, &d.elem_bpfac, bpf)) || (rc = upload(m, &d.edge_dxdy, exy)) ||
        (rc = upload(m, &d.edge_cross, ecr)) || (rc = upload(m, &d.node_tvol, tvol)))
        return rc;
    // packed members, in storage order (each member's range is the same
    // there, the storage order keeping members apart)
    d.n_members = m->n_members;
    if (m->n_members > 1) {
        std::vector<int> nm(N), em(E);
        for (int i = 0; i < N; ++i) nm[i] = nmem[nd_ref[i]];
        for (int i = 0; i < E; ++i) em[i] = emem[el_ref[i]];
        if ((rc = upload(m, &d.node_member, nm)) || (rc = upload(m, &d.elem_member, em)) ||
            (rc = upload(m, &d.member_node_off, m->member_node_off)) ||
            (rc = upload(m, &d.member_scale_area, m->member_scale_area)))
            return rc;
    }
    return FESOMC_OK;
}

// elevation family, river / open-boundary inputs, status words and the
// energy scratch: FP64 in both forms, held by the f64 view
int alloc_2d(fesomc_model *m) {
    Dev &d = m->d;
    const size_t N = d.N;
    int rc = 0;
    double **nodes[] = {&d.eta_n, &d.eta_n_1, &d.eta_n_2, &d.eta_new, &d.etaAB, &d.ssh_gp, &d.eta_jac,
                        &d.eta_jac_old};
    for (auto p : nodes) if ((rc = dalloc(m, p, N))) return rc;
    if ((rc = dalloc(m, &d.runoff, (size_t)(d.n_rivers > 0 ? d.n_rivers : 1)))) return rc;
    if ((rc = dalloc(m, &d.ob_val, (size_t)(d.nobn > 0 ? d.nobn : 1) * (m->p.Mt > 0 ? m->p.Mt : 1)))) return rc;
    if (m->p.key_atm) {
        // array_setup: mslp = P_ref (fv_main.F90:1006); qns = qsr = emp = 0 (:1050-1053)
        double **atm[] = {&d.mslp, &d.emp, &d.qsr, &d.qns};
        for (auto p : atm) if ((rc = dalloc(m, p, N))) return rc;
        std::vector<double> pref(N, kPref);
        CK(cudaMemcpy(d.mslp, pref.data(), N * sizeof(double), cudaMemcpyHostToDevice));
        if (m->p.type_swr_body == 1 && !m->p.jer_const) {
            double **jer[] = {&d.Rj, &d.aj, &d.bj};
            for (auto p : jer) if ((rc = dalloc(m, p, N))) return rc;
        }
    }
    if ((rc = dalloc(m, &d.status, 1))) return rc;
    if ((rc = dalloc(m, &d.notconv, 1))) return rc;
    if ((rc = dalloc(m, &m->d_epart, (size_t)3 * energy_parts()))) return rc;
    if ((rc = dalloc(m, &m->d_eout, 4))) return rc;
    return FESOMC_OK;
}

// 2D momentum, its forcing and the sub-cycle scratch, in the working
// precision of D
template <typename D>
int alloc_mom2d(fesomc_model *m, D &d) {
    const size_t N = d.N, E = d.E;
    int rc = 0;
    decltype(&d.mask_wd) nodes[] = {&d.mask_wd_node, &d.windx, &d.windy};
    for (auto p : nodes) if ((rc = dalloc(m, p, N))) return rc;
    decltype(&d.mask_wd) elems[] = {&d.aux_elem, &d.dmean_n, &d.U_filt_2D, &d.V_filt_2D, &d.mask_wd, &d.taux, &d.tauy};
    for (auto p : elems) if ((rc = dalloc(m, p, E))) return rc;
    decltype(&d.UAB) e2[] = {&d.U_n_2D, &d.U_n_1, &d.U_n_2, &d.UAB, &d.U_rhs_2D_3D, &d.Bar_pr_2D};
    for (auto p : e2) if ((rc = dalloc(m, p, E))) return rc;
    if ((rc = dalloc(m, &d.vel_grad, E))) return rc;
    if ((rc = dalloc(m, &d.bfric, E))) return rc;
    if ((rc = dalloc(m, &d.adv2d, (size_t)d.Ed_in)) || (rc = dalloc(m, &d.sshfl, (size_t)d.Ed))) return rc;
    if (m->p.filt_bi_2D && (rc = dalloc(m, &d.f2uv2d, E))) return rc;
    if (m->p.bih_2D && ((rc = dalloc(m, &d.b2fl, (size_t)d.Ed)) || (rc = dalloc(m, &d.b2ul, E)))) return rc;
    return FESOMC_OK;
}

// level fields and scratch of the 3D kernels, in the working precision of D
template <typename D>
int alloc_3d(fesomc_model *m, D &d) {
    const size_t N = d.N, E = d.E, L = d.L, NS = d.NS;
    int rc = 0;
    if ((rc = dalloc(m, &d.Fp, E))) return rc;
    if ((rc = dalloc(m, &d.adv3, L * (size_t)d.Ed_in))) return rc;
    if (m->p.bih_3D && ((rc = dalloc(m, &d.bihfl, L * (size_t)d.Ed)) || (rc = dalloc(m, &d.bihU, L * E)) ||
                        (rc = dalloc(m, &d.bihV, L * E))))
        return rc;
    if (m->p.filt_bi_3D && ((rc = dalloc(m, &d.f2U, L * E)) || (rc = dalloc(m, &d.f2V, L * E)))) return rc;
    decltype(&d.U_n) le[] = {&d.U_n, &d.V_n, &d.U_rhsAB, &d.V_rhsAB, &d.U_n_filt, &d.V_n_filt, &d.U_rhs, &d.V_rhs,
                             &d.U_puls, &d.V_puls, &d.vgux, &d.vguy, &d.vgvx, &d.vgvy, &d.Bar_pru, &d.Bar_prv,
                             &d.Je, &d.Ze, &d.ZBe};
    for (auto p : le) if ((rc = dalloc(m, p, L * E))) return rc;
    decltype(&d.U_n) ln[] = {&d.Unode, &d.Vnode, &d.Unode_p, &d.Vnode_p, &d.TF, &d.SF, &d.T_old, &d.S_old,
                             &d.Tclim, &d.Sclim, &d.rho_c, &d.TF_adv, &d.SF_adv, &d.Told_new, &d.Sold_new,
                             &d.ttfold, &d.stfold};
    for (auto p : ln) if ((rc = dalloc(m, p, L * N))) return rc;
    if (m->p.tracer_adv == FESOMC_TRACER_MUSCL || m->p.tracer_adv == FESOMC_TRACER_MIURA) {
        decltype(&d.U_n) lg[] = {&d.ttx, &d.tty, &d.stx, &d.sty};
        for (auto p : lg) if ((rc = dalloc(m, p, L * E))) return rc;
        decltype(&d.U_n) lgn[] = {&d.tnx, &d.tny, &d.snx, &d.sny};
        for (auto p : lgn) if ((rc = dalloc(m, p, L * N))) return rc;
        decltype(&d.mflT) fl[] = {&d.mflT, &d.mflS, &d.mflC};
        for (auto p : fl) if ((rc = dalloc(m, p, L * (size_t)d.Ed))) return rc;
    }
    if (m->p.tracer_adv == FESOMC_TRACER_MIURA) {
        if ((rc = dalloc(m, &d.tnow, L * N))) return rc;
        if ((rc = dalloc(m, &d.mask_ad, N))) return rc;
    }
    decltype(&d.U_n) nsn[] = {&d.hpressure, &d.bt, &d.snu, &d.Kv, &d.Ri, &d.tke_dissip, &d.Wvel};
    for (auto p : nsn) if ((rc = dalloc(m, p, NS * N))) return rc;
    if (m->p.ver_mix == 3) {
        decltype(&d.U_n) d3s[] = {&d.d3_pb, &d.d3_qb, &d.d3_c2, &d.d3_sn};
        for (auto p : d3s) if ((rc = dalloc(m, p, NS * N))) return rc;
    }
    if ((rc = dalloc(m, &d.Av, NS * E))) return rc;
    const size_t nm = (size_t)m->n_members;
    if ((rc = dalloc(m, &d.mm_part, (size_t)4 * nm * fesomc::f64::minmax_parts((int)nm)))) return rc;
    if ((rc = dalloc(m, &d.aver, 2 * nm))) return rc;
    return FESOMC_OK;
}

int alloc_state(fesomc_model *m) {
    int rc = alloc_2d(m);
    if (rc) return rc;
    if (m->fp32) return (rc = alloc_mom2d(m, m->d32)) ? rc : alloc_3d(m, m->d32);
    return (rc = alloc_mom2d(m, m->d)) ? rc : alloc_3d(m, m->d);
}

// FP32 form: the f32 view shares the sizes, flags, connectivity and the FP64
// elevation family with the f64 view, and holds FP32 copies of the mesh
// geometry and its own FP32 2D momentum.
template <typename TO>
int geom_f32(fesomc_model *m, const void *src, size_t n_doubles, const TO **dst) {
    std::vector<double> h(n_doubles);
    CK(cudaMemcpy(h.data(), src, n_doubles * sizeof(double), cudaMemcpyDeviceToHost));
    std::vector<float> g(n_doubles);
    for (size_t i = 0; i < n_doubles; ++i) g[i] = (float)h[i];
    float *q = nullptr;
    int rc = dalloc(m, &q, n_doubles);
    if (rc) return rc;
    CK(cudaMemcpy(q, g.data(), n_doubles * sizeof(float), cudaMemcpyHostToDevice));
    *dst = reinterpret_cast<const TO *>(q);
    return FESOMC_OK;
}

int setup_f32_view(fesomc_model *m) {
    const Dev &a = m->d;
    fesomc::f32::Dev &b = m->d32;
    b.N = a.N; b.E = a.E; b.Ed = a.Ed; b.Ed_in = a.Ed_in; b.L = a.L; b.NS = a.NS;
    b.nobn = a.nobn; b.n_rivers = a.n_rivers;
    b.elem_nodes = a.elem_nodes; b.elem_nb = a.elem_nb; b.elem_edges = a.elem_edges; b.elem_iedges = a.elem_iedges;
    b.elem_sedges = a.elem_sedges;
    b.edge_nodes = a.edge_nodes; b.edge_tri = a.edge_tri; b.edge_updn = a.edge_updn;
    b.node_eptr = a.node_eptr; b.node_eidx = a.node_eidx; b.node_nptr = a.node_nptr; b.node_nidx = a.node_nidx;
    b.node_bptr = a.node_bptr; b.node_bidx = a.node_bidx; b.node_rptr = a.node_rptr; b.node_ridx = a.node_ridx;
    b.obn_of_node = a.obn_of_node; b.index_nod2D = a.index_nod2D;
    b.n_members = a.n_members; b.node_member = a.node_member; b.elem_member = a.elem_member;
    b.member_node_off = a.member_node_off;
    const size_t N = a.N, E = a.E, Ed = a.Ed, L = a.L, NS = a.NS;
    int rc;
    if (a.member_scale_area && (rc = geom_f32(m, a.member_scale_area, a.n_members, &b.member_scale_area))) return rc;
    if ((rc = geom_f32(m, a.sig, NS, &b.sig)) || (rc = geom_f32(m, a.dsig, L, &b.dsig)) ||
        (rc = geom_f32(m, a.w_cv, 4 * E, &b.w_cv)) || (rc = geom_f32(m, a.gs_x, 4 * E, &b.gs_x)) ||
        (rc = geom_f32(m, a.gs_y, 4 * E, &b.gs_y)) || (rc = geom_f32(m, a.gv_x, 4 * E, &b.gv_x)) ||
        (rc = geom_f32(m, a.gv_y, 4 * E, &b.gv_y)) || (rc = geom_f32(m, a.elem_area, E, &b.elem_area)) ||
        (rc = geom_f32(m, a.elem_cos, E, &b.elem_cos)) || (rc = geom_f32(m, a.coriolis, E, &b.coriolis)) ||
        (rc = geom_f32(m, a.area, N, &b.area)) || (rc = geom_f32(m, a.depth, N, &b.depth)) ||
        (rc = geom_f32(m, a.ac, N, &b.ac)) || (rc = geom_f32(m, a.atp1, N, &b.atp1)) ||
        (rc = geom_f32(m, a.atp2, N, &b.atp2)) || (rc = geom_f32(m, a.elem_acc, E, &b.elem_acc)) ||
        (rc = geom_f32(m, a.elem_bpfac, E, &b.elem_bpfac)) || (rc = geom_f32(m, a.edge_dxdy, 2 * Ed, &b.edge_dxdy)) ||
        (rc = geom_f32(m, a.edge_cross, 4 * Ed, &b.edge_cross)) || (rc = geom_f32(m, a.node_tvol, N, &b.node_tvol)))
        return rc;
    return FESOMC_OK;
}

// share the FP64 elevation family, inputs and status words with the f32
// view (after alloc_state)
void share_2d(fesomc_model *m) {
    const Dev &a = m->d;
    fesomc::f32::Dev &b = m->d32;
    b.eta_n = a.eta_n; b.eta_n_1 = a.eta_n_1; b.eta_n_2 = a.eta_n_2; b.eta_new = a.eta_new; b.etaAB = a.etaAB;
    b.ssh_gp = a.ssh_gp; b.eta_jac = a.eta_jac; b.eta_jac_old = a.eta_jac_old;
    b.runoff = a.runoff; b.ob_val = a.ob_val; b.status = a.status; b.notconv = a.notconv;
    b.mslp = a.mslp; b.emp = a.emp; b.qsr = a.qsr; b.qns = a.qns; b.Rj = a.Rj; b.aj = a.aj; b.bj = a.bj;
}

template <typename D>
void set_params(D &d, const fesomc_params &p) {
    d.dt = p.dt; d.dt_2D = p.dt_2D; d.Dmin = p.Dmin; d.C_d = p.C_d; d.beta = p.beta; d.epsilon = p.epsilon;
    d.density_0 = p.density_0; d.scale_area = p.scale_area; d.snul = p.snul; d.z0b_min = p.z0b_min;
    d.z0s_min = p.z0s_min; d.Pr_num = p.Pr_num; d.beta_scale = p.beta_scale; d.cka = p.cka;
    d.tau_inv_filt = p.tau_inv_filt; d.K_hor = p.K_hor; d.Cd_bz = p.Cd_bz; d.clim_relax = p.clim_relax;
    d.relax2clim_ac = p.relax2clim_ac; d.river_salinity = p.river_salinity; d.Mt = p.Mt;
    d.mom_adv_2D = p.mom_adv_2D; d.mom_adv_3D = p.mom_adv_3D; d.vert_adv = p.vert_adv;
    d.im_vert_visc = p.im_vert_visc; d.im_vert_visc_fic = p.im_vert_visc_fic; d.fic_point = p.fic_point;
    d.tracer_adv = p.tracer_adv; d.ver_mix = p.ver_mix; d.filt_2D = p.filt_2D; d.filt_3D = p.filt_3D;
    d.wet_dry_on = p.wet_dry_on; d.key_rivers = p.key_rivers; d.TF_presence = p.TF_presence; d.cl_relax = p.cl_relax;
    d.beta_d = p.beta; d.Dmin_d = p.Dmin; d.dt_2D_d = p.dt_2D;
    d.bih_3D = p.bih_3D; d.Abh0 = p.Abh0;
    d.filt_bi_3D = p.filt_bi_3D; d.filt_bi_2D = p.filt_bi_2D; d.tau_c = p.tau_c; d.bih_2D = p.bih_2D;
    d.key_atm = p.key_atm; d.type_swr_body = p.type_swr_body; d.jer_const = p.jer_const;
    d.Rjc = p.Rjc; d.ajc = p.ajc; d.bjc = p.bjc; d.density_0_d = p.density_0;
}

// Algorithmic bytes per launch of every kernel: each array the kernel must
// read or write counted once at its element size (connectivity and geometry
// once), no credit for re-reads.  N nodes, E elements, Ed edges (Ei
// internal), L layers, NS = L+1 interfaces.
double kernel_bytes_fp64(const fesomc_model *m, const std::string &k) {
    const Dev &d = m->d;
    const double N = d.N, E = d.E, Ed = d.Ed, Ei = d.Ed_in, L = d.L, NS = d.NS;
    const double nnz_ne = (double)(2 * d.Ed);  // node->edge incidences
    if (k == "biharmonic")   // two edge passes, U_c, its gradients
        return 2 * (L * Ed * 16 + Ed * (8 + 8 + 16 + 32 + 16) + L * E * 32 + L * E * 16) + L * E * (16 + 16) +
               E * 16 + L * E * (16 + 32) + E * (16 + 16 + 64) + N * 16;
    if (k == "biharmonic_2d")   // pulsation gradients, two edge passes, U_c, its gradients
        return L * E * (16 + 32) + E * (16 + 16 + 64 + 16) + 2 * (L * Ed * 16 + Ed * 48 + L * E * 48) +
               L * E * (16 + 16) + E * 16 + L * E * (16 + 32);
    if (k == "filt2x") return L * E * (16 + 16 + 8 * 4) + E * (16 + 8) + L * E * 16;
    if (k == "filt2x_2d") return E * (16 + 16 + 8 + 16);
    if (k == "potential") return N * (16 + 8);   // coordinates in, ssh_gp out
    if (k == "bih_2d") return 2 * (Ed * (16 + 8 + 32 + 8 + 16) + E * 32 + Ed * 16) + E * (16 + 16 + 8 + 8 + 16) +
                              E * (16 + 16 + 64 + 16 + 32);
    if (k == "forcing") return (double)d.nobn * (m->p.Mt * 8 + 12 * 16) + 36 * 8 + d.n_rivers * 16.0 + 16;
    // ab3_elem (AB3 levels, w_cv, nodes; eta levels and depth; UAB, aux out)
    // and velgrad2d (UAB, neighbours, edges, gradients, cos; vel_grad out)
    if (k == "ab3_elem") return E * (48 + 32 + 16) + N * 32 + E * (16 + 8) + E * (16 + 16 + 16 + 64 + 8) + E * 32;
    // ssh_edge (edge geometry, UAB, aux; the flux out) and ssh_node (CSR,
    // the fluxes, node fields)
    if (k == "ssh_node") return N * (4 + 4 + 4 + 24 + 8 + 8 + 16) + 4 * nnz_ne + Ed * (8 + 32) + E * 24 + Ed * 16;
    // per internal edge: nodes (etaAB, depth, ac), elements (UAB, vel_grad,
    // cos), geometry; one flux pair written
    if (k == "adv2d_edge") return N * 24 + E * (16 + 32 + 8) + Ei * (8 + 8 + 32 + 16 + 16);
    // per element: 4 nodes' etaAB, depth, atp1/2, ssh_gp, eta_n, eta_new;
    // element fields read / written once; edge fluxes of its internal edges
    if (k == "u2d_elem")
        return N * 56 + E * (16 + 8 + 32 + 8 + 64 + 16 + 8 + 16 + 16 + 16 + 16 + 32 + 16 + 16 + 16 + 16) +
               Ei * 16 + E * (8 + 16 + 16 + 16 + 16);
    if (k == "rot_nodes") return N * 48;
    if (k == "pressure_col") return L * N * 16 + N * 16 + L * N * 8 + NS * N * 8;
    if (k == "bpg_elem") return NS * N * 8 + N * 48 + E * (96 + 16 + 8 + 8) + L * E * 8 + L * E * 16 + E * 32;
    if (k == "el2nodes" || k == "el2nodes_p") return L * E * 16 + N * 12 + 4 * (4.0 * E) + E * 8 + L * N * 16;
    if (k == "d3end") return L * N * 32 + NS * N * 24 + N * 40 + NS * N * 40;
    if (k == "av") return NS * N * 8 + E * 48 + NS * E * 8;
    if (k == "velgrad3d") return L * E * 16 + E * (48 + 64 + 8) + L * E * 32;
    if (k == "adv3_edge") return L * E * 48 + N * 24 + Ei * 64 + E * 8 + L * Ei * 16;
    if (k == "velrhs")
        return L * E * (48 + 24) + L * Ei * 16 + NS * N * 8 + N * 16 + E * 168 + L * E * 32;
    if (k == "implvisc") return L * E * 16 + NS * E * 8 + E * (16 + 16 + 16) + L * E * 16 + L * E * 16;
    if (k == "zero_filt") return E * 16 + E * 8 + E * 16 + E * 32;
    if (k == "puls_elem") return L * E * 16 + E * 16 + N * 24 + E * 48 + L * E * 16 + E * 8;
    if (k == "p1_edge") return L * N * 16 + N * 16 + Ei * 32 + E * 8 + L * Ei * 16;
    if (k == "p1_elem")
        return L * Ei * 16 + E * (16 + 16 + 16) + Ei * 8 + N * 8 + L * E * 8 +
               (d.filt_3D ? L * E * 16 + E * 24 : 0.0);
    if (k == "jac_swap") return N * 32;
    if (k == "update3d") return L * E * (16 + 8 + 32 + 24) + N * 24 + E * 48 + E * 32 + E * 16;
    if (k == "wvel") return N * 4 + 4 * nnz_ne + Ed * 40 + E * 16 + L * E * 24 + N * 8 + NS * N * 8;
    if (k == "minmax") return L * N * 16;
    if (k == "je_elem") return N * 16 + E * 48 + L * E * 24;
    if (k == "ab2_node") return L * N * 32 + L * N * 16;
    if (k == "miura")
        return (L * N * 24 + N * 24 + L * N * 16) + (L * N * 8 + E * 80 + L * E * 16) +
               (L * E * 16 + N * 4 + 4 * (4.0 * E) + E * 8 + L * N * 16) +
               (L * N * 40 + N * 8 + L * E * 48 + Ed * 64 + E * 8 + L * Ed * 32) +
               (L * Ed * 32 + 4 * nnz_ne + N * 4 + L * N * 16 + NS * N * 8 + L * N * 32 + L * N * 32);
    // tracer gathers: AB2 tracers (2 per node level), Je and transports per
    // element level, W per node interface, T/S of the node, edge geometry,
    // and the four outputs per node level
    if (k == "upwind_h")
        return L * N * 16 + L * E * 24 + NS * N * 8 + L * N * 16 + N * 28 + 4 * nnz_ne + Ed * 48 + L * N * 32;
    if (k == "muscl_egrad") return L * N * 16 + E * 80 + L * E * 32;
    if (k == "muscl_ngrad") return L * E * 32 + N * 4 + 4 * (4.0 * E) + E * 8 + L * N * 32;
    // edge pass: AB2 tracers of the 2 end nodes and gradients (up/down
    // elements or the node fallback), Je / transports of the 2 elements,
    // edge geometry; 3 flux pairs per (edge, level) written
    if (k == "muscl_edge") return L * N * 16 + L * E * 32 + L * N * 32 + L * E * 40 + Ed * 64 + E * 8 + L * Ed * 48;
    // node pass: flux pairs of the node's edges (each array counted once),
    // AB2 tracers, W, T/S, outputs
    if (k == "muscl_h")
        return L * Ed * 48 + 4 * nnz_ne + N * 4 + L * N * 16 + NS * N * 8 + L * N * 16 + N * 28 + L * N * 32;
    if (k == "vdiff_col") return L * N * 32 + NS * N * 8 + N * 16 + L * N * 32;
    return 0.0;
}

// In the FP32 form the 3D kernels and the 2D momentum kernels move their
// fields (almost all of their bytes) at half the size; the elevation
// kernels (ssh_node, rot_nodes, jac_swap) keep FP64 and are counted as such.
double kernel_bytes(const fesomc_model *m, const std::string &k) {
    const double b = kernel_bytes_fp64(m, k);
    if (!m->fp32) return b;
    if (k == "ssh_node" || k == "rot_nodes" || k == "jac_swap" || k == "forcing" || k == "potential") return b;
    return 0.5 * b;
}

// Runs fn() bracketed by profiling events when profiling is on.
template <typename F>
void rec(fesomc_model *m, const char *name, F fn) {
    auto &P = m->prof;
    if (!P.on) { fn(); return; }
    int k = -1;
    for (size_t i = 0; i < P.names.size(); ++i)
        if (P.names[i] == name) { k = (int)i; break; }
    if (k < 0) {
        P.names.push_back(name);
        P.bytes.push_back(kernel_bytes(m, name));
        P.ms.push_back(0.0);
        P.count.push_back(0);
        k = (int)P.names.size() - 1;
    }
    if (P.used + 2 > P.ev.size()) {
        for (int i = 0; i < 64; ++i) {
            cudaEvent_t e;
            cudaEventCreate(&e);
            P.ev.push_back(e);
        }
    }
    cudaEventRecord(P.ev[P.used], m->stream);
    fn();
    cudaEventRecord(P.ev[P.used + 1], m->stream);
    P.rec_kernel.push_back(k);
    P.used += 2;
}

// The kernel sequence of one internal step (oce_timestep case(3)).  The 2D
// sub-cycle kernels always run on the FP64 view; the 3D kernels on the view
// of the model's form (K3).
// device forcing view of the model (valid after fesomc_gpu_set_device_forcing)
ForcingDev forcing_view(const fesomc_model *m) {
    ForcingDev f{};
    const Dev &d = m->d;
    f.nobn = d.nobn;
    f.n_rivers = d.n_rivers;
    f.Mt = m->p.Mt;
    f.restart = m->p.restart;
    f.tides_on = m->p.TF_presence && d.nobn > 0;
    f.rivers_on = m->p.key_rivers && d.n_rivers > 0 && m->d_runoff_base != nullptr;
    f.river_ramp = m->river_ramp;
    f.dt = m->p.dt;
    f.dt_2D = m->p.dt_2D;
    f.time_jd0 = m->p.time_jd0;
    f.clock = m->d_clock;
    f.ampt = m->d_ampt;
    f.fazt = m->d_fazt;
    f.harm = m->d_harm;
    f.runoff_base = m->d_runoff_base;
    f.ob_val = d.ob_val;
    f.runoff = d.runoff;
    return f;
}

int enqueue_step(fesomc_model *m, double ff) {
    const Dev &d = m->d;
    const fesomc::f32::Dev &q = m->d32;
    const bool f = m->fp32;
    cudaStream_t s = m->stream;
    int n = 0;
#define K3(fn, ...) (f ? fesomc::f32::fn(q, ##__VA_ARGS__) : fesomc::f64::fn(d, ##__VA_ARGS__))
#define K3E2N(a, b, c, e) (f ? fesomc::f32::launch_el2nodes(q, q.a, q.b, q.c, q.e, s) \
                             : fesomc::f64::launch_el2nodes(d, d.a, d.b, d.c, d.e, s))
    if (m->dev_forcing) {
        rec(m, "forcing", [&] { launch_forcing(forcing_view(m), s); });
        n += 2;
    }
    if (m->dev_atm) {
        // sbc_do (fv_main.F90:419), before the step, from the previous
        // step's surface velocity and temperature
        const AtmDev a{m->d_atm_a, m->d_atm_b, m->d_clock, m->d_tau_node, m->atm_net_flux, m->atm_prec_coef};
        rec(m, "atm_fluxes", [&] { fesomc::f64::launch_atm(d, a, s); });
        n += 2;
    }
    if (m->p.T_potential) {
        // potential at the head of oce_timestep (fv_main.F90:1899)
        PotentialDev pd{};
        pd.N = d.N;
        pd.time_jd0 = m->p.time_jd0;
        for (int k = 0; k < m->p.n_harm; ++k)
            if (m->p.harm_index[k] >= 0 && m->p.harm_index[k] < 11) pd.ath[m->p.harm_index[k]] = 1.0;
        pd.clock = m->d_clock;
        pd.coord = m->d_coord;
        pd.ssh_gp = f ? q.ssh_gp : d.ssh_gp;
        rec(m, "potential", [&] { launch_potential(pd, s); });
        n += 1;
    }
    rec(m, "pressure_col", [&] { K3(launch_pressure_col, s); });
    rec(m, "bpg_elem", [&] { K3(launch_bpg_elem, s); });
    n += 2;
    rec(m, "el2nodes", [&] { K3E2N(U_n, V_n, Unode, Vnode); });
    n += 1;
    if (d.ver_mix == 3 && m->lc_on) {
        // learned closure: inputs, envelope test and fallback list; the
        // network on every column; its viscosity where it applies and the
        // plain closure on the listed columns, or (judge step) the plain
        // closure everywhere, compared with the network
        const LcView &c = m->lcv;
        CK(cudaMemsetAsync(c.count, 0, sizeof(unsigned long long), s));
        rec(m, "lc_features", [&] { K3(launch_lc_features, c, s); });
        if (m->lc_bf16) rec(m, "lc_infer_tc", [&] { lc_forward_tc(m->lc, c.X, d.N, c.Y, s); });
        else rec(m, "lc_infer", [&] { lc_forward_full(m->lc, c.X, d.N, c.Y, m->lc_bufA, m->lc_bufB, s); });
        n += 5;
        if (m->lc_judge_now) {
            rec(m, "d3end", [&] { K3(launch_d3end, s); });
            rec(m, "lc_judge", [&] { K3(launch_lc_judge, c, s); });
        } else {
            rec(m, "lc_apply", [&] { K3(launch_lc_apply, c, s); });
            rec(m, "d3end_list", [&] { K3(launch_d3end_list, c.list, c.count, s); });
        }
        rec(m, "av", [&] { K3(launch_av, s); });
        n += 3;
    } else if (d.ver_mix == 3) {
        rec(m, "d3end", [&] { K3(launch_d3end, s); });
        if (m->lc_harvest_now) { rec(m, "lc_harvest", [&] { K3(launch_lc_harvest, m->lcv, s); }); n += 3; }
        rec(m, "av", [&] { K3(launch_av, s); });
        n += 2;
    }
    rec(m, "velgrad3d", [&] { K3(launch_velgrad3d, s); });
    n += 1;
    if (d.mom_adv_3D == 1) { rec(m, "adv3_edge", [&] { K3(launch_adv3_edge, s); }); n += 1; }
    if (d.filt_bi_3D) { rec(m, "filt2x", [&] { K3(launch_filt2x, s); }); n += 1; }
    if (d.bih_3D) { rec(m, "biharmonic", [&] { K3(launch_bih, s); }); n += 4; }
    rec(m, "velrhs", [&] { K3(launch_velrhs, ff, s); });
    n += 1;
    if (d.im_vert_visc || d.im_vert_visc_fic) { rec(m, "implvisc", [&] { K3(launch_implvisc, s); }); n += 1; }
    rec(m, "zero_filt", [&] { K3(launch_zero_filt, s); });
    n += 1;
    for (int sub = 0; sub < d.Mt; ++sub) {
        rec(m, "ab3_elem", [&] { K3(launch_ab3_elem, s); });
        rec(m, "ssh_node", [&] { K3(launch_ssh_node, sub, s); });
        n += 4;
        if (sub == 0) {
            rec(m, "puls_elem", [&] { K3(launch_puls_elem, s); });
            rec(m, "el2nodes_p", [&] { K3E2N(U_puls, V_puls, Unode_p, Vnode_p); });
            rec(m, "p1_edge", [&] { K3(launch_p1_edge, s); });
            if (d.bih_3D) { rec(m, "biharmonic_2d", [&] { K3(launch_bih_puls, s); }); n += 5; }
            rec(m, "p1_elem", [&] { K3(launch_p1_elem, s); });
            n += 4;
        }
        if (d.mom_adv_2D == 2) { rec(m, "adv2d_edge", [&] { K3(launch_adv2d_edge, s); }); n += 1; }
        if (d.filt_bi_2D) { rec(m, "filt2x_2d", [&] { K3(launch_filt2x_2d, s); }); n += 1; }
        if (d.bih_2D) { rec(m, "bih_2d", [&] { K3(launch_bih_2d, s); }); n += 4; }
        rec(m, "u2d_elem", [&] { K3(launch_u2d_elem, s); });
        rec(m, "rot_nodes", [&] { K3(launch_rot_nodes, s); });
        n += 2;
    }
    rec(m, "jac_swap", [&] { launch_jac_swap(d, s); });
    rec(m, "update3d", [&] { K3(launch_update3d, 1.0 / (double)d.Mt, s); });
    rec(m, "wvel", [&] { K3(launch_wvel, s); });
    if (m->ext_range) rec(m, "minmax", [&] { K3(launch_aver_from_range, m->d_ext_range, s); });
    else rec(m, "minmax", [&] { K3(launch_minmax, s); });
    n += m->ext_range ? 4 : 5;
    if (d.tracer_adv != FESOMC_TRACER_MIURA) { rec(m, "ab2_node", [&] { K3(launch_ab2, s); }); n += 1; }
    if (d.tracer_adv == FESOMC_TRACER_MIURA) { rec(m, "miura", [&] { K3(launch_miura, s); }); n += 5; }
    else if (d.tracer_adv == FESOMC_TRACER_MUSCL) {
        rec(m, "muscl_egrad", [&] { K3(launch_muscl_egrad, s); });
        rec(m, "muscl_ngrad", [&] { K3(launch_muscl_ngrad, s); });
        rec(m, "muscl_edge", [&] { K3(launch_muscl_edge, s); });
        rec(m, "muscl_h", [&] { K3(launch_muscl_h, s); });
        n += 4;
    }
    else { rec(m, "upwind_h", [&] { K3(launch_upwind, s); }); n += 1; }
    rec(m, "vdiff_col", [&] { K3(launch_vdiff, s); });
    n += 1;
#undef K3E2N
#undef K3
    m->launches_per_step = n;
    CK(cudaGetLastError());
    return FESOMC_OK;
}

// Open-boundary elevation for the Mt sub-steps of the coming internal step
// (compute_ssh_rhs_elem, fv_average_dynamic.F90:190-216), on the host with
// the reference formula; 'time' is the internal-step time in seconds.
// Harmonics with a zero amplitude are skipped: their term is a signed zero,
// and adding it to the partial sum (which starts at +0) changes no bit.
void ob_values(const fesomc_model *m, double time, double time_jd, double *out) {
    const fesomc_params &p = m->p;
    const int nobn = m->d.nobn;
    for (int sub = 0; sub < p.Mt; ++sub) {
        const double time_2D = time + p.dt_2D * (sub + 1);
        for (int q = 0; q < nobn; ++q) {
            double v = 0.0;
            for (int j = 0; j < 12; ++j) {
                const double amp = m->amp_factor[j] * m->ampt[(size_t)nobn * j + q];
                if (amp == 0.0) continue;
                v = v + amp *
                            fesomc_cos((time_2D - p.time_jd0 * 86400.0) * 2.0 * kPi / (kHarmPeriod[j] * 3600.0) -
                                     (m->fazt[(size_t)nobn * j + q] + m->phy_factor[j]));
            }
            if (!p.restart)
                if (time_jd - p.time_jd0 < 10.0) v = v * (time_jd - p.time_jd0) / 10.0;
            out[(size_t)sub * nobn + q] = v;
        }
    }
}

int upload_step_inputs(fesomc_model *m, double time, double time_jd) {
    const int nobn = m->d.nobn, nr = m->d.n_rivers;
    const bool need_ob = m->p.TF_presence && nobn > 0;
    const bool need_r = m->p.key_rivers && nr > 0 && m->runoff_dirty;
    const bool need_clock = (m->p.T_potential != 0 || m->dev_atm) && !m->dev_forcing;
    if (!need_ob && !need_r && !need_clock) return FESOMC_OK;
    const int i = m->stage_i;
    m->stage_i ^= 1;
    CK(cudaEventSynchronize(m->stage_ev[i]));
    double *h = m->h_stage[i];
    size_t off = 0;
    if (need_ob) {
        if (m->pre_valid && m->pre_time_jd == time_jd) std::memcpy(h, m->h_pre.data(), sizeof(double) * nobn * m->p.Mt);
        else ob_values(m, time, time_jd, h);
        CK(cudaMemcpyAsync(m->d.ob_val, h, sizeof(double) * nobn * m->p.Mt, cudaMemcpyHostToDevice, m->stream));
        off += (size_t)nobn * m->p.Mt;
    }
    if (need_r) {
        std::memcpy(h + off, m->h_runoff, sizeof(double) * nr);
        CK(cudaMemcpyAsync(m->d.runoff, h + off, sizeof(double) * nr, cudaMemcpyHostToDevice, m->stream));
        m->runoff_dirty = false;
        off += (size_t)nr;
    }
    if (need_clock) {
        // the step's time_jd for the tidal potential kernel
        h[off] = time_jd;
        CK(cudaMemcpyAsync(m->d_clock, h + off, sizeof(double), cudaMemcpyHostToDevice, m->stream));
    }
    CK(cudaEventRecord(m->stage_ev[i], m->stream));
    return FESOMC_OK;
}

int collect_status(fesomc_model *m) {
    Dev &d = m->d;
    CK(cudaMemcpyAsync(m->h_status, d.status, sizeof(unsigned), cudaMemcpyDeviceToHost, m->stream));
    CK(cudaMemcpyAsync(m->h_notconv, d.notconv, sizeof(int), cudaMemcpyDeviceToHost, m->stream));
    CK(cudaMemsetAsync(d.status, 0, sizeof(unsigned), m->stream));
    CK(cudaMemsetAsync(d.notconv, 0, sizeof(int), m->stream));
    CK(cudaStreamSynchronize(m->stream));
    m->status_acc |= *m->h_status;
    m->notconv_acc += *m->h_notconv;
    return FESOMC_OK;
}

int status_code(unsigned st) {
    if (st & FESOMC_ST_NONFINITE) return FESOMC_ENONFINITE;
    if (st & FESOMC_ST_NEGSALT) return FESOMC_ENEGSALT;
    if (st & FESOMC_ST_LOWTEMP) return FESOMC_ELOWTEMP;
    return FESOMC_OK;
}

int run_steps(fesomc_model *m, int nsteps) {
    // per-node Jerlov water types must have come with the forcing
    if (m->d.Rj && !m->have_jer) return FESOMC_ESTATE;
    for (int k = 0; k < nsteps; ++k) {
        // time update of the main loop (fv_main.F90:400-401)
        m->time_jd = m->time_jd + m->p.dt / 86400.0;
        const double time = m->time_jd * 86400.0;
        int rc = m->dev_forcing ? FESOMC_OK : upload_step_inputs(m, time, m->time_jd);
        if (rc) return rc;
        // learned closure: every lc_judge_every-th step is a judge step
        if (m->lc_on) {
            m->lc_steps += 1;
            m->lc_judge_now = m->lc_judge_every > 0 && m->lc_steps % m->lc_judge_every == 0;
            if (m->lc_judge_now) m->lc_judges += 1;
        }
        const bool eager = m->lc_judge_now || m->lc_harvest_now;
        if (m->lfirst) {
            // first call of compute_vel_rhs: AB2 factor 1 (fv_3D_vel.F90:124-128)
            rc = enqueue_step(m, 1.0);
            if (rc) return rc;
            m->lfirst = 0;
        } else if (eager) {
            rc = enqueue_step(m, 1.5 + m->p.epsilon);
            if (rc) return rc;
        } else if (m->use_graph) {
            if (!m->graph) {
                cudaGraph_t g;
                CK(cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeThreadLocal));
                rc = enqueue_step(m, 1.5 + m->p.epsilon);
                cudaError_t ce = cudaStreamEndCapture(m->stream, &g);
                if (rc) return rc;
                CK(ce);
                CK(cudaGraphInstantiate(&m->graph, g, 0));
                CK(cudaGraphDestroy(g));
            }
            CK(cudaGraphLaunch(m->graph, m->stream));
        } else {
            rc = enqueue_step(m, 1.5 + m->p.epsilon);
            if (rc) return rc;
        }
        m->launches += m->launches_per_step;
        if (!m->dev_forcing && m->p.TF_presence && m->d.nobn > 0) {
            // the next step's open-boundary table, while this step runs
            const double tj = m->time_jd + m->p.dt / 86400.0;
            m->h_pre.resize((size_t)m->d.nobn * m->p.Mt);
            ob_values(m, tj * 86400.0, tj, m->h_pre.data());
            m->pre_time_jd = tj;
            m->pre_valid = true;
        }
    }
    return FESOMC_OK;
}

// tide harmonics of the device forcing from the host copies
int upload_tides(fesomc_model *m) {
    const size_t nobn = (size_t)m->d.nobn;
    if (nobn) {
        CK(cudaMemcpy(m->d_ampt, m->ampt.data(), nobn * 12 * sizeof(double), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(m->d_fazt, m->fazt.data(), nobn * 12 * sizeof(double), cudaMemcpyHostToDevice));
    }
    double h[36];
    for (int j = 0; j < 12; ++j) {
        h[j] = m->amp_factor[j];
        h[12 + j] = m->phy_factor[j];
        h[24 + j] = kHarmPeriod[j];
    }
    CK(cudaMemcpy(m->d_harm, h, sizeof(h), cudaMemcpyHostToDevice));
    return FESOMC_OK;
}

}  // namespace

extern "C" {

namespace {
// A packed member table: ranges that start at 0, grow strictly and end at
// the mesh's counts, and connectivity that never crosses from one member to
// another (elements' nodes, edges' nodes and elements, nodes' elements).
bool members_valid(const fesomc_mesh *msh, const fesomc_members *mb) {
    const int n = mb->n, N = msh->nod2D, E = msh->elem2D;
    if (n < 1 || !mb->node_off || !mb->elem_off || !mb->scale_area) return false;
    if (mb->node_off[0] != 0 || mb->elem_off[0] != 0 || mb->node_off[n] != N || mb->elem_off[n] != E) return false;
    for (int k = 0; k < n; ++k) {
        if (mb->node_off[k + 1] <= mb->node_off[k] || mb->elem_off[k + 1] <= mb->elem_off[k]) return false;
        if (!(mb->scale_area[k] > 0.0) || !std::isfinite(mb->scale_area[k])) return false;
    }
    std::vector<int> nm(N), em(E);
    for (int k = 0; k < n; ++k) {
        for (int i = mb->node_off[k]; i < mb->node_off[k + 1]; ++i) nm[i] = k;
        for (int i = mb->elem_off[k]; i < mb->elem_off[k + 1]; ++i) em[i] = k;
    }
    auto node_in = [&](int32_t ref1, int k) { return ref1 >= 1 && ref1 <= N && nm[ref1 - 1] == k; };
    auto elem_in = [&](int32_t ref1, int k) { return ref1 >= 1 && ref1 <= E && em[ref1 - 1] == k; };
    for (int e = 0; e < E; ++e)
        for (int j = 0; j < 4; ++j) {
            if (!node_in(msh->elem2D_nodes[4 * e + j], em[e])) return false;
            const int32_t nb = msh->elem_neighbors[4 * e + j];
            if (nb > 0 && !elem_in(nb, em[e])) return false;
        }
    for (int ed = 0; ed < msh->edge2D; ++ed) {
        const int32_t a = msh->edge_nodes[2 * ed];
        if (a < 1 || a > N) return false;
        const int k = nm[a - 1];
        if (!node_in(msh->edge_nodes[2 * ed + 1], k) || !elem_in(msh->edge_tri[2 * ed], k)) return false;
        if (msh->edge_tri[2 * ed + 1] > 0 && !elem_in(msh->edge_tri[2 * ed + 1], k)) return false;
        if (msh->edge_up_dn_tri)
            for (int j = 0; j < 2; ++j)
                if (msh->edge_up_dn_tri[2 * ed + j] > 0 && !elem_in(msh->edge_up_dn_tri[2 * ed + j], k)) return false;
    }
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < msh->nod_in_elem2D_num[i]; ++j)
            if (!elem_in(msh->nod_in_elem2D[(size_t)msh->nod_in_elem2D_max * i + j], nm[i])) return false;
    return true;
}
}  // namespace

int fesomc_gpu_init(const fesomc_mesh *mesh, const fesomc_params *par, const fesomc_state *st, fesomc_model **out) {
    return fesomc_gpu_init_packed(mesh, par, st, nullptr, out);
}

int fesomc_gpu_init_packed(const fesomc_mesh *mesh, const fesomc_params *par, const fesomc_state *st,
                           const fesomc_members *members, fesomc_model **out) {
    if (!mesh || !par || !st || !out) return FESOMC_EINVAL;
    *out = nullptr;
    if (mesh->nsigma < 5 || mesh->nsigma > 127 || mesh->nod2D < 3 || mesh->elem2D < 1) return FESOMC_EINVAL;
    if (par->Mt < 1 || par->dt <= 0.0 || par->dt_2D <= 0.0) return FESOMC_EINVAL;
    if (par->ver_mix != 3 && par->ver_mix != 0) return FESOMC_EINVAL;
    if (par->tracer_adv != FESOMC_TRACER_UPWIND && par->tracer_adv != FESOMC_TRACER_MUSCL &&
        par->tracer_adv != FESOMC_TRACER_MIURA)
        return FESOMC_EINVAL;
    if (par->tracer_adv == FESOMC_TRACER_MUSCL && !mesh->edge_up_dn_tri) return FESOMC_EINVAL;
    if (par->cl_solid_boder_relax) return FESOMC_EINVAL;
    if (par->mom_adv_2D != 2 && par->mom_adv_2D != 0) return FESOMC_EINVAL;
    if (par->mom_adv_3D != 1 && par->mom_adv_3D != 0) return FESOMC_EINVAL;
    if (par->fp32_form != 0 && par->fp32_form != 1) return FESOMC_EINVAL;
    if (par->bih_3D != 0 && par->bih_3D != 1) return FESOMC_EINVAL;
    if (par->bih_3D && !std::isfinite(par->Abh0)) return FESOMC_EINVAL;
    if ((par->filt_bi_3D != 0 && par->filt_bi_3D != 1) || (par->filt_bi_2D != 0 && par->filt_bi_2D != 1) ||
        (par->bih_2D != 0 && par->bih_2D != 1))
        return FESOMC_EINVAL;
    if (par->bih_2D && !std::isfinite(par->Abh0)) return FESOMC_EINVAL;
    if (par->T_potential != 0 && par->T_potential != 1) return FESOMC_EINVAL;
    if (par->npes < 0 || par->npes > 1) return FESOMC_EINVAL;   // one rank: no halo exchange
    if (par->sfc_order != 0 && par->sfc_order != 1) return FESOMC_EINVAL;
    if (par->sfc_order && !mesh->coord_nod2D) return FESOMC_EINVAL;
    if (par->key_atm != 0 && par->key_atm != 1) return FESOMC_EINVAL;
    if (par->key_atm && (par->type_swr_body < 1 || par->type_swr_body > 2 ||   // fv_read_run.F90:799-803
                         (par->jer_const != 0 && par->jer_const != 1)))
        return FESOMC_EINVAL;
    if (!st->eta_n || !st->TF || !st->SF || !st->U_n || !st->V_n) return FESOMC_EINVAL;
    if (members && !members_valid(mesh, members)) return FESOMC_EINVAL;
    fesomc_model *m = new (std::nothrow) fesomc_model();
    if (!m) return FESOMC_ENOMEM;
    if (members && members->n > 1) {
        m->n_members = members->n;
        m->member_node_off.assign(members->node_off, members->node_off + members->n + 1);
        m->member_elem_off.assign(members->elem_off, members->elem_off + members->n + 1);
        m->member_scale_area.assign(members->scale_area, members->scale_area + members->n);
    }
    m->p = *par;
    m->fp32 = par->fp32_form == 1;
    set_params(m->d, *par);
    set_params(m->d32, *par);
    int rc = FESOMC_OK;
    auto fail = [&](int code) {
        fesomc_gpu_finalize(m);
        return code;
    };
    // the launch checks below read the thread's last CUDA error: start from
    // a clean one (a non-sticky error of an earlier, unrelated call is not ours)
    (void)cudaGetLastError();
    if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(FESOMC_ECUDA);
    if ((rc = build_mesh(m, mesh))) return fail(rc);
    if (m->fp32 && (rc = setup_f32_view(m))) return fail(rc);
    if ((rc = alloc_state(m))) return fail(rc);
    if (m->fp32) share_2d(m);
    // kernels whose shared-memory scratch scales with the level count
    if (m->fp32) {
        const fesomc::f32::Dev &q = m->d32;
        if (fesomc::f32::config_d3end(q) || fesomc::f32::config_vdiff(q) || fesomc::f32::config_p1(q) ||
            fesomc::f32::config_columns(q))
            return fail(FESOMC_EINVAL);
    } else if (config_d3end(m->d) || config_vdiff(m->d) || config_p1(m->d) || config_columns(m->d)) {
        return fail(FESOMC_EINVAL);
    }
    const size_t nobn = (size_t)(mesh->nobn > 0 ? mesh->nobn : 0);
    m->ampt.assign(nobn * 12, 0.0);
    m->fazt.assign(nobn * 12, 0.0);
    for (int j = 0; j < 12; ++j) { m->amp_factor[j] = 1.0; m->phy_factor[j] = 0.0; }
    m->stage_len = nobn * (size_t)par->Mt + (size_t)(mesh->n_rivers > 0 ? mesh->n_rivers : 0) + 8;
    for (int i = 0; i < 2; ++i) {
        if (cudaMallocHost(&m->h_stage[i], m->stage_len * sizeof(double)) != cudaSuccess) return fail(FESOMC_ENOMEM);
        if (cudaEventCreateWithFlags(&m->stage_ev[i], cudaEventDisableTiming) != cudaSuccess) return fail(FESOMC_ECUDA);
    }
    if (cudaMallocHost(&m->h_runoff, sizeof(double) * (mesh->n_rivers + 1)) != cudaSuccess) return fail(FESOMC_ENOMEM);
    std::memset(m->h_runoff, 0, sizeof(double) * (mesh->n_rivers + 1));
    if (cudaMallocHost(&m->h_status, sizeof(unsigned) * 2) != cudaSuccess) return fail(FESOMC_ENOMEM);
    if (par->T_potential) {
        if (!mesh->coord_nod2D) return fail(FESOMC_EINVAL);
        std::vector<double2> lonlat((size_t)mesh->nod2D);
        for (int i = 0; i < mesh->nod2D; ++i)
            lonlat[i] = make_double2(mesh->coord_nod2D[2 * (size_t)i], mesh->coord_nod2D[2 * (size_t)i + 1]);
        if ((rc = upload(m, &m->d_coord, lonlat)) || (rc = dalloc(m, &m->d_clock, 1))) return fail(rc);
        if (m->perm) {   // coordinates in storage order
            if ((rc = perm_buf(m, lonlat.size() * sizeof(double2)))) return fail(rc);
            if (cudaMemcpyAsync(m->d_perm_buf, lonlat.data(), lonlat.size() * sizeof(double2), cudaMemcpyHostToDevice,
                                m->stream) != cudaSuccess)
                return fail(FESOMC_ECUDA);
            permute_from(m, ENT_NODE, (const double *)m->d_perm_buf, (double *)m->d_coord, 2 * lonlat.size(), m->stream);
            if (cudaStreamSynchronize(m->stream) != cudaSuccess) return fail(FESOMC_ECUDA);
        }
    }
    if (cudaMallocHost(&m->h_notconv, sizeof(int) * 2) != cudaSuccess) return fail(FESOMC_ENOMEM);
    // state upload (all groups that are provided)
    if ((rc = fesomc_gpu_sync_from_host(m, FESOMC_F_ALL, st))) return fail(rc);
    if (!st->mask_wd) {
        std::vector<double> ones(mesh->elem2D, 1.0);
        void *dev = m->fp32 ? (void *)m->d32.mask_wd : (void *)m->d.mask_wd;
        if ((rc = field_from_host(m, dev, m->fp32, ones.size(), ones.data(), ENT_ELEM))) return fail(rc);
    }
    if (!st->mask_wd_node) {
        std::vector<double> ones(mesh->nod2D, 1.0);
        void *dev = m->fp32 ? (void *)m->d32.mask_wd_node : (void *)m->d.mask_wd_node;
        if ((rc = field_from_host(m, dev, m->fp32, ones.size(), ones.data(), ENT_NODE))) return fail(rc);
    }
    // jacobian state before the main loop: both calls see the initial eta
    if (cudaMemcpy(m->d.eta_jac, m->d.eta_n, sizeof(double) * mesh->nod2D, cudaMemcpyDeviceToDevice) ||
        cudaMemcpy(m->d.eta_jac_old, m->d.eta_n, sizeof(double) * mesh->nod2D, cudaMemcpyDeviceToDevice))
        return fail(FESOMC_ECUDA);
    if (m->fp32) fesomc::f32::launch_je(m->d32, m->stream);
    else launch_je(m->d, m->stream);
    if (cudaGetLastError() != cudaSuccess) return fail(FESOMC_ECUDA);
    m->lfirst = st->lfirst;
    m->time_jd = st->time_jd;
    if (cudaDeviceSynchronize() != cudaSuccess) return fail(FESOMC_ECUDA);
    *out = m;
    return FESOMC_OK;
}

int fesomc_gpu_set_forcing(fesomc_model *m, const fesomc_forcing *fin) {
    if (!m || !fin) return FESOMC_EINVAL;
    // with sbc_do on the device the step forms the winds, the stress and the
    // surface fluxes itself
    fesomc_forcing fa = *fin;
    if (m->dev_atm) fa.taux = fa.tauy = fa.windx = fa.windy = fa.mslp = fa.emp = fa.qsr = fa.qns = nullptr;
    const fesomc_forcing *f = &fa;
    Dev &d = m->d;
    const size_t N = d.N, E = d.E, L = d.L;
    cudaStream_t s = m->stream;
    // large fields are copied synchronously with respect to the stream so the
    // caller may reuse its buffers on return
    int rc = FESOMC_OK;
    if (!m->fp32 && m->perm) {
        CK(cudaStreamSynchronize(s));
        if (f->taux && (rc = field_from_host(m, d.taux, false, E, f->taux, ENT_ELEM))) return rc;
        if (f->tauy && (rc = field_from_host(m, d.tauy, false, E, f->tauy, ENT_ELEM))) return rc;
        if (f->windx && (rc = field_from_host(m, d.windx, false, N, f->windx, ENT_NODE))) return rc;
        if (f->windy && (rc = field_from_host(m, d.windy, false, N, f->windy, ENT_NODE))) return rc;
    } else if (!m->fp32) {
        if (f->taux) CK(cudaMemcpyAsync(d.taux, f->taux, E * 8, cudaMemcpyHostToDevice, s));
        if (f->tauy) CK(cudaMemcpyAsync(d.tauy, f->tauy, E * 8, cudaMemcpyHostToDevice, s));
        if (f->windx) CK(cudaMemcpyAsync(d.windx, f->windx, N * 8, cudaMemcpyHostToDevice, s));
        if (f->windy) CK(cudaMemcpyAsync(d.windy, f->windy, N * 8, cudaMemcpyHostToDevice, s));
    } else if (f->taux || f->tauy || f->windx || f->windy) {
        // FP32 form: converted on the host, written while the stream is idle
        const fesomc::f32::Dev &q = m->d32;
        CK(cudaStreamSynchronize(s));
        if (f->taux && (rc = field_from_host(m, q.taux, true, E, f->taux, ENT_ELEM))) return rc;
        if (f->tauy && (rc = field_from_host(m, q.tauy, true, E, f->tauy, ENT_ELEM))) return rc;
        if (f->windx && (rc = field_from_host(m, q.windx, true, N, f->windx, ENT_NODE))) return rc;
        if (f->windy && (rc = field_from_host(m, q.windy, true, N, f->windy, ENT_NODE))) return rc;
    }
    if (f->Tclim || f->Sclim) CK(cudaStreamSynchronize(s));
    if (f->Tclim &&
        (rc = field_from_host(m, m->fp32 ? (void *)m->d32.Tclim : (void *)d.Tclim, m->fp32, L * N, f->Tclim, ENT_NODE)))
        return rc;
    if (f->Sclim &&
        (rc = field_from_host(m, m->fp32 ? (void *)m->d32.Sclim : (void *)d.Sclim, m->fp32, L * N, f->Sclim, ENT_NODE)))
        return rc;
    if (f->taux || f->tauy || f->windx || f->windy || f->Tclim || f->Sclim) CK(cudaStreamSynchronize(s));
    if (d.mslp) {   // key_atm: FP64 node fields in both forms
        const double *src[] = {f->mslp, f->emp, f->qsr, f->qns, f->Rj, f->aj, f->bj};
        double *dst[] = {d.mslp, d.emp, d.qsr, d.qns, d.Rj, d.aj, d.bj};
        CK(cudaStreamSynchronize(s));
        for (int k = 0; k < 7; ++k)
            if (src[k] && dst[k] && (rc = field_from_host(m, dst[k], false, N, src[k], ENT_NODE))) return rc;
        if (d.Rj && f->Rj && f->aj && f->bj) m->have_jer = true;
        CK(cudaStreamSynchronize(s));
    }
    if (f->runoff_rivers && d.n_rivers > 0) {
        std::memcpy(m->h_runoff, f->runoff_rivers, sizeof(double) * d.n_rivers);
        m->runoff_dirty = true;
    }
    const size_t nobn = (size_t)d.nobn;
    if ((f->ampt && nobn) || (f->fazt && nobn) || f->amp_factor || f->phy_factor) m->pre_valid = false;
    if (f->ampt && nobn) std::memcpy(m->ampt.data(), f->ampt, nobn * 12 * 8);
    if (f->fazt && nobn) std::memcpy(m->fazt.data(), f->fazt, nobn * 12 * 8);
    if (f->amp_factor) std::memcpy(m->amp_factor, f->amp_factor, 12 * 8);
    if (f->phy_factor) std::memcpy(m->phy_factor, f->phy_factor, 12 * 8);
    if (m->dev_forcing && ((f->ampt && nobn) || (f->fazt && nobn) || f->amp_factor || f->phy_factor)) {
        CK(cudaStreamSynchronize(s));
        if ((rc = upload_tides(m))) return rc;
    }
    return FESOMC_OK;
}

int fesomc_gpu_set_device_forcing(fesomc_model *m, const double *runoff_base, int32_t river_ramp) {
    if (!m) return FESOMC_EINVAL;
    const Dev &d = m->d;
    const bool rivers = m->p.key_rivers && d.n_rivers > 0;
    if (rivers && !runoff_base) return FESOMC_EINVAL;
    int rc;
    CK(cudaStreamSynchronize(m->stream));
    if (!m->d_clock && (rc = dalloc(m, &m->d_clock, 1))) return rc;
    if (!m->d_ampt) {
        const size_t nobn = (size_t)(d.nobn > 0 ? d.nobn : 1);
        if ((rc = dalloc(m, &m->d_ampt, 12 * nobn)) ||
            (rc = dalloc(m, &m->d_fazt, 12 * nobn)) || (rc = dalloc(m, &m->d_harm, 36)) ||
            (rc = dalloc(m, &m->d_runoff_base, (size_t)(d.n_rivers > 0 ? d.n_rivers : 1))))
            return rc;
    }
    if ((rc = upload_tides(m))) return rc;
    if (rivers) CK(cudaMemcpy(m->d_runoff_base, runoff_base, sizeof(double) * d.n_rivers, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(m->d_clock, &m->time_jd, sizeof(double), cudaMemcpyHostToDevice));
    m->river_ramp = river_ramp != 0;
    if (!m->dev_forcing && m->graph) {
        // the captured step has no forcing kernels: capture again
        cudaGraphExecDestroy(m->graph);
        m->graph = nullptr;
    }
    m->dev_forcing = true;
    return FESOMC_OK;
}

int fesomc_gpu_step(fesomc_model *m, int32_t n_dt) {
    (void)n_dt;
    if (!m) return FESOMC_ESTATE;
    int rc = run_steps(m, 1);
    if (rc) return rc;
    if ((rc = collect_status(m))) return rc;
    return status_code(m->status_acc);
}

int fesomc_gpu_run(fesomc_model *m, int32_t n_dt0, int32_t nsteps) {
    (void)n_dt0;
    if (!m || nsteps < 0) return FESOMC_EINVAL;
    int rc = run_steps(m, nsteps);
    if (rc) return rc;
    if ((rc = collect_status(m))) return rc;
    return status_code(m->status_acc);
}

int fesomc_gpu_sync_to_host(fesomc_model *m, uint32_t mask, fesomc_state *st) {
    if (!m || !st) return FESOMC_EINVAL;
    CK(cudaStreamSynchronize(m->stream));
    for (const FieldRef &f : field_table(m)) {
        double *h = st->*(f.host);
        int rc;
        if ((f.group & mask) && h && (rc = field_to_host(m, f, h))) return rc;
    }
    st->lfirst = m->lfirst;
    st->time_jd = m->time_jd;
    return FESOMC_OK;
}

int fesomc_gpu_sync_from_host(fesomc_model *m, uint32_t mask, const fesomc_state *st) {
    if (!m || !st) return FESOMC_EINVAL;
    CK(cudaStreamSynchronize(m->stream));
    for (const FieldRef &f : field_table(m)) {
        const double *h = st->*(f.host);
        int rc;
        if ((f.group & mask) && h && (rc = field_from_host(m, f.dev, f.f32, f.count, h, f.ent))) return rc;
    }
    if (mask == FESOMC_F_ALL) {
        m->lfirst = st->lfirst;
        m->time_jd = st->time_jd;
        if (m->d_clock) CK(cudaMemcpy(m->d_clock, &m->time_jd, sizeof(double), cudaMemcpyHostToDevice));
        // a restart: the jacobian state from the restart elevation, as the
        // reference's jacobian call after reading a restart (fv_main.F90:364);
        // a running model holds the same at every step boundary
        const size_t N = (size_t)m->d.N;
        CK(cudaMemcpy(m->d.eta_jac, m->d.eta_n, sizeof(double) * N, cudaMemcpyDeviceToDevice));
        CK(cudaMemcpy(m->d.eta_jac_old, m->d.eta_n, sizeof(double) * N, cudaMemcpyDeviceToDevice));
        if (m->fp32) fesomc::f32::launch_je(m->d32, m->stream);
        else launch_je(m->d, m->stream);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(m->stream));
    }
    return FESOMC_OK;
}

// ---- halo exchange of a decomposed mesh on the device ----------------------
// A plan holds a list of the model's nodes and elements (device indices);
// pack gathers every field of the restart set (the field table's order,
// each entity's values consecutive, FP32 fields widened) for those entities
// into a device buffer of doubles, unpack scatters such a buffer back.
int fesomc_gpu_halo_plan(fesomc_model *m, int32_t n_nodes, const int32_t *nodes, int32_t n_elems,
                         const int32_t *elems, fesomc_halo **out) {
    if (!m || !out || n_nodes < 0 || n_elems < 0 || (n_nodes && !nodes) || (n_elems && !elems)) return FESOMC_EINVAL;
    *out = nullptr;
    const int N = m->d.N, E = m->d.E;
    // reference -> device index (the storage order's inverse)
    std::vector<int> nd(N), el(E);
    if (m->perm) {
        std::vector<int> nref(N), eref(E);
        CK(cudaMemcpy(nref.data(), m->d_nd_ref, sizeof(int) * N, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(eref.data(), m->d_el_ref, sizeof(int) * E, cudaMemcpyDeviceToHost));
        for (int i = 0; i < N; ++i) nd[nref[i]] = i;
        for (int i = 0; i < E; ++i) el[eref[i]] = i;
    } else {
        for (int i = 0; i < N; ++i) nd[i] = i;
        for (int i = 0; i < E; ++i) el[i] = i;
    }
    std::vector<int> hn(n_nodes), he(n_elems);
    for (int i = 0; i < n_nodes; ++i) {
        if (nodes[i] < 0 || nodes[i] >= N) return FESOMC_EINVAL;
        hn[i] = nd[nodes[i]];
    }
    for (int i = 0; i < n_elems; ++i) {
        if (elems[i] < 0 || elems[i] >= E) return FESOMC_EINVAL;
        he[i] = el[elems[i]];
    }
    fesomc_halo *h = new fesomc_halo();
    h->n_nodes = n_nodes;
    h->n_elems = n_elems;
    for (const FieldRef &f : field_table(m))
        h->count += (long long)(f.ent == ENT_NODE ? n_nodes : n_elems) * (long long)(f.count / ents(m, f.ent));
    cudaError_t e = cudaMalloc(&h->d_range, 4 * sizeof(double));
    if (e == cudaSuccess && n_nodes) e = cudaMalloc(&h->d_nodes, sizeof(int) * n_nodes);
    if (e == cudaSuccess && n_elems) e = cudaMalloc(&h->d_elems, sizeof(int) * n_elems);
    if (e == cudaSuccess && n_nodes) e = cudaMemcpy(h->d_nodes, hn.data(), sizeof(int) * n_nodes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && n_elems) e = cudaMemcpy(h->d_elems, he.data(), sizeof(int) * n_elems, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        fesomc_gpu_halo_free(h);
        return e == cudaErrorMemoryAllocation ? FESOMC_ENOMEM : FESOMC_ECUDA;
    }
    *out = h;
    return FESOMC_OK;
}

int fesomc_gpu_halo_size(const fesomc_halo *h, int64_t *count) {
    if (!h || !count) return FESOMC_EINVAL;
    *count = h->count;
    return FESOMC_OK;
}

int fesomc_gpu_halo_pack(fesomc_model *m, const fesomc_halo *h, double *buf) {
    if (!m || !h || (h->count && !buf)) return FESOMC_EINVAL;
    long long off = 0;
    for (const FieldRef &f : field_table(m)) {
        const int n = f.ent == ENT_NODE ? h->n_nodes : h->n_elems;
        const int w = (int)(f.count / ents(m, f.ent));
        const int *idx = f.ent == ENT_NODE ? h->d_nodes : h->d_elems;
        if (n) {
            const int g = grid_for((long long)n * w, 256);
            if (f.f32) k_halo_gather<<<g, 256, 0, m->stream>>>((const float *)f.dev, w, idx, n, buf + off);
            else k_halo_gather<<<g, 256, 0, m->stream>>>((const double *)f.dev, w, idx, n, buf + off);
        }
        off += (long long)n * w;
    }
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(m->stream));
    return FESOMC_OK;
}

int fesomc_gpu_halo_unpack(fesomc_model *m, const fesomc_halo *h, const double *buf) {
    if (!m || !h || (h->count && !buf)) return FESOMC_EINVAL;
    long long off = 0;
    for (const FieldRef &f : field_table(m)) {
        const int n = f.ent == ENT_NODE ? h->n_nodes : h->n_elems;
        const int w = (int)(f.count / ents(m, f.ent));
        const int *idx = f.ent == ENT_NODE ? h->d_nodes : h->d_elems;
        if (n) {
            const int g = grid_for((long long)n * w, 256);
            if (f.f32) k_halo_scatter<<<g, 256, 0, m->stream>>>((float *)f.dev, w, idx, n, buf + off);
            else k_halo_scatter<<<g, 256, 0, m->stream>>>((double *)f.dev, w, idx, n, buf + off);
        }
        off += (long long)n * w;
    }
    // the jacobian state follows the elevation, as after a full upload: a
    // running model holds eta_jac = eta_n at every step boundary
    const size_t N = (size_t)m->d.N;
    CK(cudaMemcpyAsync(m->d.eta_jac, m->d.eta_n, sizeof(double) * N, cudaMemcpyDeviceToDevice, m->stream));
    CK(cudaMemcpyAsync(m->d.eta_jac_old, m->d.eta_n, sizeof(double) * N, cudaMemcpyDeviceToDevice, m->stream));
    if (m->fp32) fesomc::f32::launch_je(m->d32, m->stream);
    else launch_je(m->d, m->stream);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(m->stream));
    return FESOMC_OK;
}

int fesomc_gpu_halo_range(fesomc_model *m, const fesomc_halo *h, double *range) {
    if (!m || !h || !range || h->n_nodes < 1) return FESOMC_EINVAL;
    const FieldRef *tf = nullptr, *sf = nullptr;
    const std::vector<FieldRef> table = field_table(m);
    for (const FieldRef &f : table) {
        if (f.host == &fesomc_state::TF) tf = &f;
        if (f.host == &fesomc_state::SF) sf = &f;
    }
    const int w = (int)(tf->count / ents(m, ENT_NODE));
    if (tf->f32) k_halo_range<<<1, 256, 0, m->stream>>>((const float *)tf->dev, (const float *)sf->dev, w, h->d_nodes, h->n_nodes, h->d_range);
    else k_halo_range<<<1, 256, 0, m->stream>>>((const double *)tf->dev, (const double *)sf->dev, w, h->d_nodes, h->n_nodes, h->d_range);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(range, h->d_range, 4 * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
    CK(cudaStreamSynchronize(m->stream));
    return FESOMC_OK;
}

void fesomc_gpu_halo_free(fesomc_halo *h) {
    if (!h) return;
    cudaFree(h->d_nodes);
    cudaFree(h->d_elems);
    cudaFree(h->d_range);
    delete h;
}

int fesomc_gpu_snapshot_begin(fesomc_model *m, uint32_t mask, fesomc_state *st) {
    if (!m || !st) return FESOMC_EINVAL;
    if (m->snap_pending) return FESOMC_ESTATE;
    if (!m->copy_stream) {
        CK(cudaStreamCreateWithFlags(&m->copy_stream, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&m->snap_taken, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&m->snap_done, cudaEventDisableTiming));
    }
    const std::vector<FieldRef> table = field_table(m);
    if (m->snap_bufs.size() < table.size()) {
        m->snap_bufs.resize(table.size(), {nullptr, nullptr});
        m->snap_bytes.resize(table.size(), 0);
    }
    m->snaps.clear();
    // device-to-device copies on the step stream: the state after every step
    // enqueued so far, taken without waiting for the host
    for (size_t i = 0; i < table.size(); ++i) {
        const FieldRef &f = table[i];
        double *dst = st->*(f.host);
        if (!(f.group & mask) || !dst) continue;
        const size_t bytes = f.count * (f.f32 ? sizeof(float) : sizeof(double));
        if (m->snap_bytes[i] != bytes) {
            unsigned char *dc = nullptr;
            int rc = dalloc(m, &dc, bytes);
            if (rc) return rc;
            float *hp = nullptr;
            if (f.f32 && cudaMallocHost(&hp, bytes) != cudaSuccess) return FESOMC_ENOMEM;
            m->snap_bufs[i] = {dc, hp};
            m->snap_bytes[i] = bytes;
        }
        if (!f.f32) {
            // the caller's array receives the copy directly: page-lock it once
            bool known = false;
            for (auto &r : m->registered) known |= (r.first == (void *)dst && r.second >= bytes);
            if (!known) {
                // an array that shares pages with one registered already
                // cannot be registered; its copy then runs unlocked (the
                // driver stages it), which is slower but correct
                if (cudaHostRegister(dst, f.count * sizeof(double), cudaHostRegisterDefault) == cudaSuccess)
                    m->registered.push_back({dst, f.count * sizeof(double)});
                else
                    (void)cudaGetLastError();
            }
        }
        if (!m->perm)
            CK(cudaMemcpyAsync(m->snap_bufs[i].first, f.dev, bytes, cudaMemcpyDeviceToDevice, m->stream));
        else if (f.f32)   // the copy in reference order
            unpermute_to(m, f.ent, (const float *)f.dev, (float *)m->snap_bufs[i].first, f.count, m->stream);
        else
            unpermute_to(m, f.ent, (const double *)f.dev, (double *)m->snap_bufs[i].first, f.count, m->stream);
        m->snaps.push_back({dst, m->snap_bufs[i].first, f.f32 ? m->snap_bufs[i].second : nullptr, f.count});
    }
    CK(cudaEventRecord(m->snap_taken, m->stream));
    // device-to-host copies on the copy stream, overlapping the next steps
    CK(cudaStreamWaitEvent(m->copy_stream, m->snap_taken, 0));
    for (const auto &sn : m->snaps) {
        if (sn.pinned32)
            CK(cudaMemcpyAsync(sn.pinned32, sn.dev_copy, sn.count * sizeof(float), cudaMemcpyDeviceToHost,
                               m->copy_stream));
        else
            CK(cudaMemcpyAsync(sn.dst, sn.dev_copy, sn.count * sizeof(double), cudaMemcpyDeviceToHost,
                               m->copy_stream));
    }
    CK(cudaEventRecord(m->snap_done, m->copy_stream));
    m->snap_state = st;
    m->snap_time_jd = m->time_jd;
    m->snap_lfirst = m->lfirst;
    m->snap_pending = true;
    return FESOMC_OK;
}

int fesomc_gpu_snapshot_end(fesomc_model *m) {
    if (!m) return FESOMC_EINVAL;
    if (!m->snap_pending) return FESOMC_ESTATE;
    CK(cudaEventSynchronize(m->snap_done));
    m->snap_pending = false;
    for (const auto &sn : m->snaps)
        if (sn.pinned32)
            for (size_t i = 0; i < sn.count; ++i) sn.dst[i] = (double)sn.pinned32[i];
    m->snap_state->time_jd = m->snap_time_jd;
    m->snap_state->lfirst = m->snap_lfirst;
    return FESOMC_OK;
}

int fesomc_gpu_energy(fesomc_model *m, double *eout) {
    if (!m || !eout) return FESOMC_EINVAL;
    if (m->fp32) fesomc::f32::launch_energy(m->d32, m->d_epart, m->d_eout, m->stream);
    else launch_energy(m->d, m->d_epart, m->d_eout, m->stream);
    m->launches += 2;
    double h[3];
    CK(cudaMemcpyAsync(h, m->d_eout, 3 * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
    CK(cudaStreamSynchronize(m->stream));
    *eout = (h[0] + h[1]) / h[2];
    return FESOMC_OK;
}

int fesomc_gpu_last_status(fesomc_model *m, uint32_t *status, int32_t *notconv) {
    if (!m) return FESOMC_EINVAL;
    if (status) *status = m->status_acc | (m->notconv_acc ? FESOMC_ST_NOTCONV : 0u);
    if (notconv) *notconv = m->notconv_acc;
    m->status_acc = 0;
    m->notconv_acc = 0;
    return FESOMC_OK;
}

int fesomc_gpu_finalize(fesomc_model *m) {
    if (!m) return FESOMC_OK;
    if (m->lc && m->lc->stream == m->stream) m->lc->stream = nullptr;
    if (m->stream) cudaStreamSynchronize(m->stream);
    if (m->graph) cudaGraphExecDestroy(m->graph);
    for (cudaEvent_t e : m->prof.ev) cudaEventDestroy(e);
    for (void *p : m->allocs) cudaFree(p);
    for (int i = 0; i < 2; ++i) {
        if (m->h_stage[i]) cudaFreeHost(m->h_stage[i]);
        if (m->stage_ev[i]) cudaEventDestroy(m->stage_ev[i]);
    }
    if (m->copy_stream) cudaStreamSynchronize(m->copy_stream);
    for (auto &b : m->snap_bufs)
        if (b.second) cudaFreeHost(b.second);
    for (auto &r : m->registered) cudaHostUnregister(r.first);
    if (m->snap_taken) cudaEventDestroy(m->snap_taken);
    if (m->snap_done) cudaEventDestroy(m->snap_done);
    if (m->copy_stream) cudaStreamDestroy(m->copy_stream);
    if (m->h_runoff) cudaFreeHost(m->h_runoff);
    if (m->h_status) cudaFreeHost(m->h_status);
    if (m->h_notconv) cudaFreeHost(m->h_notconv);
    if (m->stream) cudaStreamDestroy(m->stream);
    delete m;
    return FESOMC_OK;
}

const char *fesomc_gpu_error_string(int code) {
    switch (code) {
        case FESOMC_OK: return "ok";
        case FESOMC_EINVAL: return "invalid argument or unsupported option";
        case FESOMC_ENOMEM: return "out of memory";
        case FESOMC_ECUDA: return "CUDA runtime error";
        case FESOMC_ESTATE: return "call out of order";
        case FESOMC_ENEGSALT: return "negative salinity, time resolution is insufficient";
        case FESOMC_ELOWTEMP: return "temperature below -3 C, time resolution is insufficient";
        case FESOMC_ENONFINITE: return "non-finite value in the prognostic state";
        case FESOMC_ENOTCONV: return "d3_end did not converge in 200 iterations";
        case FESOMC_EMESH: return "inconsistent element node list";
        default: return "unknown error";
    }
}

int fesomc_gpu_time_run(fesomc_model *m, int32_t nsteps, double *ms) {
    if (!m || nsteps < 0 || !ms) return FESOMC_EINVAL;
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    CK(cudaStreamSynchronize(m->stream));
    CK(cudaEventRecord(a, m->stream));
    int rc = run_steps(m, nsteps);
    if (rc) return rc;
    CK(cudaEventRecord(b, m->stream));
    CK(cudaEventSynchronize(b));
    float f = 0.f;
    CK(cudaEventElapsedTime(&f, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    *ms = f;
    if ((rc = collect_status(m))) return rc;
    return status_code(m->status_acc);
}

int fesomc_gpu_profile(fesomc_model *m, int32_t nsteps, int32_t max_kernels, int32_t *n_kernels, char *names,
                       double *ms_per_launch, double *bytes_per_launch, int64_t *launches) {
    if (!m || nsteps < 1 || !n_kernels || !names || !ms_per_launch || !bytes_per_launch || !launches)
        return FESOMC_EINVAL;
    auto &P = m->prof;
    P.on = true;
    P.names.clear(); P.bytes.clear(); P.ms.clear(); P.count.clear(); P.rec_kernel.clear();
    P.used = 0;
    const bool g = m->use_graph;
    m->use_graph = false;
    int rc = run_steps(m, nsteps);
    m->use_graph = g;
    P.on = false;
    if (rc) return rc;
    CK(cudaStreamSynchronize(m->stream));
    for (size_t r = 0; r < P.rec_kernel.size(); ++r) {
        float f = 0.f;
        CK(cudaEventElapsedTime(&f, P.ev[2 * r], P.ev[2 * r + 1]));
        P.ms[P.rec_kernel[r]] += f;
        P.count[P.rec_kernel[r]] += 1;
    }
    const int nk = (int)P.names.size() < max_kernels ? (int)P.names.size() : max_kernels;
    for (int k = 0; k < nk; ++k) {
        std::memset(names + 32 * k, 0, 32);
        std::strncpy(names + 32 * k, P.names[k].c_str(), 31);
        ms_per_launch[k] = P.ms[k] / (double)P.count[k];
        bytes_per_launch[k] = P.bytes[k];
        launches[k] = P.count[k];
    }
    *n_kernels = nk;
    if ((rc = collect_status(m))) return rc;
    return status_code(m->status_acc);
}

int fesomc_ensemble_run(fesomc_model *const *members, int32_t n, int32_t nsteps, double *ms, int32_t *status) {
    if (!members || n <= 0 || nsteps < 0) return FESOMC_EINVAL;
    for (int i = 0; i < n; ++i) {
        if (!members[i]) return FESOMC_EINVAL;
        for (int j = 0; j < i; ++j)
            if (members[j] == members[i]) return FESOMC_EINVAL;
    }
    cudaEvent_t fork = nullptr, join = nullptr;
    std::vector<cudaEvent_t> done;
    auto release = [&] {
        if (fork) cudaEventDestroy(fork);
        if (join) cudaEventDestroy(join);
        for (cudaEvent_t e : done)
            if (e) cudaEventDestroy(e);
    };
    cudaStream_t s0 = members[0]->stream;
    if (ms) {
        // start from idle streams, then fork every member stream from s0
        for (int i = 0; i < n; ++i) CK(cudaStreamSynchronize(members[i]->stream));
        if (cudaEventCreate(&fork) != cudaSuccess || cudaEventCreate(&join) != cudaSuccess) {
            release();
            return FESOMC_ECUDA;
        }
        done.assign(n, nullptr);
        for (int i = 1; i < n; ++i)
            if (cudaEventCreateWithFlags(&done[i], cudaEventDisableTiming) != cudaSuccess) {
                release();
                return FESOMC_ECUDA;
            }
        CK(cudaEventRecord(fork, s0));
        for (int i = 1; i < n; ++i) CK(cudaStreamWaitEvent(members[i]->stream, fork, 0));
    }
    // one internal step of every member per round: no member's host-side
    // staging wait holds back the others' enqueues
    for (int k = 0; k < nsteps; ++k)
        for (int i = 0; i < n; ++i) {
            const int rc = run_steps(members[i], 1);
            if (rc) {
                release();
                return rc;
            }
        }
    if (ms) {
        for (int i = 1; i < n; ++i) {
            CK(cudaEventRecord(done[i], members[i]->stream));
            CK(cudaStreamWaitEvent(s0, done[i], 0));
        }
        CK(cudaEventRecord(join, s0));
        CK(cudaEventSynchronize(join));
        float f = 0.f;
        CK(cudaEventElapsedTime(&f, fork, join));
        *ms = f;
    }
    release();
    int first = FESOMC_OK;
    for (int i = 0; i < n; ++i) {
        int rc = collect_status(members[i]);
        if (rc) return rc;
        rc = status_code(members[i]->status_acc);
        if (status) status[i] = rc;
        if (first == FESOMC_OK) first = rc;
    }
    return first;
}

// ---- launch-shape knobs -----------------------------------------------------
namespace {
struct KnobInfo {
    const char *name;      // the kernel (or kernel group) the knob shapes
    const char *records;   // the fesomc_gpu_profile records that time it
    int def;               // default threads per block (0: column entities per block)
};
const KnobInfo kKnobs[fesomc::kTuneKnobs] = {
    {"velrhs", "velrhs", 256}, {"velgrad3d", "velgrad3d", 256}, {"adv3_edge", "adv3_edge", 256},
    {"puls_elem", "puls_elem", 256}, {"el2nodes", "el2nodes,el2nodes_p", 256}, {"p1_edge", "p1_edge", 256},
    {"ab3_elem", "ab3_elem", 256}, {"velgrad2d", "ab3_elem", 256}, {"ssh_edge", "ssh_node", 256},
    {"ssh_node", "ssh_node", 256}, {"adv2d_edge", "adv2d_edge", 256}, {"u2d_elem", "u2d_elem", 128},
    {"rot_nodes", "rot_nodes", 256}, {"zero_filt", "zero_filt", 256}, {"ab2_node", "ab2_node", 256},
    {"muscl_egrad", "muscl_egrad", 256}, {"muscl_ngrad", "muscl_ngrad", 256}, {"muscl_edge", "muscl_edge", 256},
    {"muscl_h", "muscl_h", 128}, {"upwind_h", "upwind_h", 128}, {"av", "av", 256},
    {"columns", "pressure_col,bpg_elem,update3d,wvel", 0},
    {"d3end_arrays", "d3end,d3end_list", 1},
    {"vdiff_form", "vdiff_col", 3},
    {"implvisc_form", "implvisc", 2},
};
int default_columns(int L) { const int b = 1024 / L; return b > 16 ? 16 : b; }
// knobs that pick a form or a count rather than threads per block
bool form_knob(int k) {
    return k == fesomc::TK_COLUMNS || k == fesomc::TK_D3END || k == fesomc::TK_VDIFF || k == fesomc::TK_IMPLVISC;
}
void drop_graph(fesomc_model *m);
int copy_str(const char *src, char *dst, int32_t len) {
    if (!dst) return FESOMC_OK;
    if (len < 1 || (int32_t)std::strlen(src) >= len) return FESOMC_EINVAL;
    std::strcpy(dst, src);
    return FESOMC_OK;
}
}  // namespace

int fesomc_gpu_set_tracer_range(fesomc_model *m, const double *range) {
    if (!m) return FESOMC_EINVAL;
    if (!range) {
        if (m->ext_range) {
            drop_graph(m);
            m->ext_range = false;
        }
        return FESOMC_OK;
    }
    if (m->n_members > 1 || !(range[0] <= range[1]) || !(range[2] <= range[3])) return FESOMC_EINVAL;
    if (!m->d_ext_range) {
        const int rc = dalloc(m, &m->d_ext_range, 4);
        if (rc) return rc;
    }
    // ordered after the steps already enqueued, which read the previous range
    CK(cudaMemcpyAsync(m->d_ext_range, range, 4 * sizeof(double), cudaMemcpyHostToDevice, m->stream));
    CK(cudaStreamSynchronize(m->stream));
    if (!m->ext_range) {
        drop_graph(m);   // the captured step computes its own range
        m->ext_range = true;
    }
    return FESOMC_OK;
}

int fesomc_gpu_set_atm_fields(fesomc_model *m, const double *coef_a, const double *coef_b, int32_t net_flux,
                              double prec_coef) {
    if (!m || !coef_a || !coef_b || !m->p.key_atm || m->fp32 || !(prec_coef != 0.0)) return FESOMC_EINVAL;
    const size_t N = (size_t)m->d.N;
    int rc;
    CK(cudaStreamSynchronize(m->stream));
    if (!m->d_atm_a) {
        if ((rc = dalloc(m, &m->d_atm_a, 8 * N)) || (rc = dalloc(m, &m->d_atm_b, 8 * N)) ||
            (rc = dalloc(m, &m->d_tau_node, 2 * N)))
            return rc;
    }
    if (!m->d_clock) {
        if ((rc = dalloc(m, &m->d_clock, 1))) return rc;
        CK(cudaMemcpy(m->d_clock, &m->time_jd, sizeof(double), cudaMemcpyHostToDevice));
    }
    // reference order [node][8] -> the storage order
    if ((rc = field_from_host(m, m->d_atm_a, false, 8 * N, coef_a, ENT_NODE)) ||
        (rc = field_from_host(m, m->d_atm_b, false, 8 * N, coef_b, ENT_NODE)))
        return rc;
    m->atm_net_flux = net_flux;
    m->atm_prec_coef = prec_coef;
    if (!m->dev_atm) {
        drop_graph(m);   // the captured step has no surface-flux kernels
        m->dev_atm = true;
    }
    return FESOMC_OK;
}

int fesomc_gpu_tune_knobs(void) { return fesomc::kTuneKnobs; }

int fesomc_gpu_tune_knob(int32_t k, char *name, int32_t name_len, char *records, int32_t records_len) {
    if (k < 0 || k >= fesomc::kTuneKnobs) return FESOMC_EINVAL;
    int rc = copy_str(kKnobs[k].name, name, name_len);
    return rc ? rc : copy_str(kKnobs[k].records, records, records_len);
}

int fesomc_gpu_tune_get(fesomc_model *m, int32_t *values, int32_t *limits) {
    if (!m || (!values && !limits)) return FESOMC_EINVAL;
    int lim[fesomc::kTuneKnobs];
    for (int k = 0; k < fesomc::kTuneKnobs; ++k) lim[k] = 1024;
    fesomc::f64::tune_limits_baroclinic(lim); fesomc::f64::tune_limits_barotropic(lim);
    fesomc::f64::tune_limits_tracer(lim); fesomc::f64::tune_limits_mixing(lim);
    fesomc::f32::tune_limits_baroclinic(lim); fesomc::f32::tune_limits_barotropic(lim);
    fesomc::f32::tune_limits_tracer(lim); fesomc::f32::tune_limits_mixing(lim);
    lim[fesomc::TK_COLUMNS] = 1024 / m->d.L < 32 ? 1024 / m->d.L : 32;
    lim[fesomc::TK_D3END] = 6;
    lim[fesomc::TK_VDIFF] = 3;
    lim[fesomc::TK_IMPLVISC] = 2;
    for (int k = 0; k < fesomc::kTuneKnobs; ++k) {
        if (values) {
            const int v = m->d.tune[k];
            values[k] = v > 0 ? v : (kKnobs[k].def > 0 ? kKnobs[k].def : default_columns(m->d.L));
        }
        if (limits)
            limits[k] = form_knob(k) ? lim[k] : (lim[k] / 32) * 32;
    }
    return FESOMC_OK;
}

int fesomc_gpu_tune_set(fesomc_model *m, const int32_t *values) {
    if (!m || !values) return FESOMC_EINVAL;
    int32_t lim[fesomc::kTuneKnobs];
    int rc = fesomc_gpu_tune_get(m, nullptr, lim);
    if (rc) return rc;
    for (int k = 0; k < fesomc::kTuneKnobs; ++k) {
        const int v = values[k];
        if (v < 0 || v > lim[k]) return FESOMC_EINVAL;
        if (!form_knob(k) && v != 0 && (v < 32 || v % 32 != 0)) return FESOMC_EINVAL;
    }
    drop_graph(m);   // the captured step holds the old launch shapes
    for (int k = 0; k < fesomc::kTuneKnobs; ++k) m->d.tune[k] = m->d32.tune[k] = values[k];
    // the column kernels' shared memory follows their entities per block
    const int bad = m->fp32 ? fesomc::f32::config_columns(m->d32) : fesomc::f64::config_columns(m->d);
    return bad ? FESOMC_EINVAL : FESOMC_OK;
}

// ---- learned vertical-mixing closure ---------------------------------------
struct fesomc_closure {
    fesomc::LcNet *net = nullptr;
};

namespace {
constexpr int kLcBatch = 8192;

// the per-column buffers of model m for closure c (made once per pairing)
int lc_model_buffers(fesomc_model *m, fesomc_closure *c) {
    LcNet *n = c->net;
    LcView &v = m->lcv;
    const int W = std::max(n->IN, n->OUT);
    v.NS = n->NS;
    v.IN = n->IN;
    v.OUT = n->OUT;
    v.mu_x = n->stats;
    v.sd_x = n->stats + W;
    v.mu_y = n->stats + 2 * W;
    v.sd_y = n->stats + 3 * W;
    v.lo_x = n->stats + 4 * W;
    v.hi_x = n->stats + 5 * W;
    v.lo_y = n->stats + 6 * W;
    v.hi_y = n->stats + 7 * W;
    v.hx = n->hx;
    v.hy = n->hy;
    v.hcap = n->hcap;
    v.hcount = n->hcount;
    if (m->lc_owner == c) return FESOMC_OK;
    const size_t N = m->d.N;
    int rc;
    if ((rc = dalloc(m, &v.X, N * n->IN)) || (rc = dalloc(m, &v.Y, N * n->OUT)) || (rc = dalloc(m, &v.flag, N)) ||
        (rc = dalloc(m, &v.list, N)) || (rc = dalloc(m, &v.count, 1)) || (rc = dalloc(m, &v.acc, 4)) ||
        (rc = dalloc(m, &v.judge, 3)) || (rc = dalloc(m, &v.blk, (N + kLcHarvestBlock - 1) / kLcHarvestBlock)))
        return rc;
    m->lc_bufA = m->lc_bufB = nullptr;   // FP32 inference activations: made when first needed
    m->lc_owner = c;
    return FESOMC_OK;
}

int lc_fp32_buffers(fesomc_model *m) {
    if (m->lc_bufA) return FESOMC_OK;
    const size_t N = m->d.N;
    int rc;
    if ((rc = dalloc(m, &m->lc_bufA, N * kLcHidden)) || (rc = dalloc(m, &m->lc_bufB, N * kLcHidden))) return rc;
    return FESOMC_OK;
}

void drop_graph(fesomc_model *m) {
    if (m->graph) {
        cudaStreamSynchronize(m->stream);
        cudaGraphExecDestroy(m->graph);
        m->graph = nullptr;
    }
}
}  // namespace

int fesomc_closure_create(int32_t nsigma, int64_t capacity, uint64_t seed, fesomc_closure **out) {
    if (!out || nsigma < 5 || nsigma > 32 || capacity < 0 || capacity >= (1LL << 31)) return FESOMC_EINVAL;
    *out = nullptr;
    fesomc_closure *c = new (std::nothrow) fesomc_closure();
    if (!c) return FESOMC_ENOMEM;
    int rc = 0;
    c->net = lc_create(nsigma, capacity, seed, kLcBatch, nullptr, &rc);
    if (!c->net) {
        delete c;
        return rc ? rc : FESOMC_ENOMEM;
    }
    *out = c;
    return FESOMC_OK;
}

void fesomc_closure_free(fesomc_closure *c) {
    if (!c) return;
    cudaDeviceSynchronize();
    lc_free(c->net);
    delete c;
}

int fesomc_closure_info(const fesomc_closure *c, int64_t *harvested, int64_t *nparams, int32_t *n_in, int32_t *n_out) {
    if (!c) return FESOMC_EINVAL;
    unsigned long long h = 0;
    CK(cudaMemcpy(&h, c->net->hcount, sizeof(h), cudaMemcpyDeviceToHost));
    if (harvested) *harvested = (int64_t)std::min<unsigned long long>(h, (unsigned long long)c->net->hcap);
    if (nparams) *nparams = c->net->np;
    if (n_in) *n_in = c->net->IN;
    if (n_out) *n_out = c->net->OUT;
    return FESOMC_OK;
}

int fesomc_closure_harvest(fesomc_closure *c, fesomc_model *m, int32_t nsteps, int32_t every) {
    if (!c || !m || nsteps < 0 || every < 1) return FESOMC_EINVAL;
    if (c->net->NS != m->d.NS || m->lc_on || m->p.ver_mix != 3) return FESOMC_ESTATE;
    int rc = lc_model_buffers(m, c);
    if (rc) return rc;
    for (int k = 0; k < nsteps; ++k) {
        m->lc_harvest_now = (k + 1) % every == 0;
        rc = run_steps(m, 1);
        m->lc_harvest_now = false;
        if (rc) return rc;
    }
    if ((rc = collect_status(m))) return rc;
    return status_code(m->status_acc);
}

int fesomc_closure_fit(fesomc_closure *c) {
    if (!c) return FESOMC_EINVAL;
    return lc_fit_stats(c->net);
}

int fesomc_closure_train(fesomc_closure *c, int32_t epochs, int32_t batch, float lr, uint64_t seed, float *losses) {
    if (!c || !(lr > 0.0f)) return FESOMC_EINVAL;
    return lc_train(c->net, epochs, batch, lr, seed, losses);
}

int fesomc_closure_params(fesomc_closure *c, float *get, const float *set) {
    if (!c) return FESOMC_EINVAL;
    const size_t b = sizeof(float) * (size_t)c->net->np;
    if (set) CK(cudaMemcpy(c->net->params, set, b, cudaMemcpyHostToDevice));
    if (get) CK(cudaMemcpy(get, c->net->params, b, cudaMemcpyDeviceToHost));
    return FESOMC_OK;
}

int fesomc_closure_norm(fesomc_closure *c, float *get, const float *set) {
    if (!c) return FESOMC_EINVAL;
    const size_t b = sizeof(float) * kLcStatRows * (size_t)std::max(c->net->IN, c->net->OUT);
    if (set) CK(cudaMemcpy(c->net->stats, set, b, cudaMemcpyHostToDevice));
    if (get) CK(cudaMemcpy(get, c->net->stats, b, cudaMemcpyDeviceToHost));
    return FESOMC_OK;
}

int fesomc_closure_forward(fesomc_closure *c, const float *X, int64_t n, float *Y, int32_t bf16) {
    if (!c || !X || !Y || n < 1) return FESOMC_EINVAL;
    LcNet *net = c->net;
    if (bf16 && !lc_tc_supported(net)) return FESOMC_EINVAL;
    if (bf16 && !net->tc_ready) {
        int rc = lc_tc_prepare(net);
        if (rc) return rc;
    }
    float *dx = nullptr, *dy = nullptr;
    if (cudaMalloc(&dx, sizeof(float) * n * net->IN) != cudaSuccess) return FESOMC_ENOMEM;
    if (cudaMalloc(&dy, sizeof(float) * n * net->OUT) != cudaSuccess) { cudaFree(dx); return FESOMC_ENOMEM; }
    int rc = FESOMC_OK;
    if (cudaMemcpy(dx, X, sizeof(float) * n * net->IN, cudaMemcpyHostToDevice) != cudaSuccess) rc = FESOMC_ECUDA;
    if (!rc) rc = bf16 ? lc_forward_tc(net, dx, n, dy, nullptr) : lc_forward(net, dx, n, dy);
    if (!rc && bf16) {
        unsigned int err = 0;
        if (cudaMemcpy(&err, net->tc_err, sizeof(err), cudaMemcpyDeviceToHost) != cudaSuccess) rc = FESOMC_ECUDA;
        else if (err) rc = FESOMC_ECUDA;
    }
    if (!rc && cudaMemcpy(Y, dy, sizeof(float) * n * net->OUT, cudaMemcpyDeviceToHost) != cudaSuccess) rc = FESOMC_ECUDA;
    cudaFree(dx);
    cudaFree(dy);
    return rc;
}

int fesomc_closure_grad(fesomc_closure *c, const float *X, const float *T, int32_t n, double *loss, float *grads) {
    if (!c || !X || !T || !loss || n < 1 || n > c->net->Bmax) return FESOMC_EINVAL;
    LcNet *net = c->net;
    CK(cudaMemcpy(net->Xb, X, sizeof(float) * (size_t)n * net->IN, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(net->Tb, T, sizeof(float) * (size_t)n * net->OUT, cudaMemcpyHostToDevice));
    int rc = lc_grad(net, net->Xb, net->Tb, n, loss);
    if (rc) return rc;
    if (grads) CK(cudaMemcpy(grads, net->grads, sizeof(float) * net->np, cudaMemcpyDeviceToHost));
    return FESOMC_OK;
}

namespace {
// deterministic pseudo-random normalised inputs for the timing entry point
__global__ void k_lc_fill(long long n, float *x, unsigned long long seed) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        unsigned long long z = (unsigned long long)i * 0x9E3779B97F4A7C15ULL + seed;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        z ^= z >> 31;
        x[i] = (float)((double)(z >> 11) * (1.0 / 9007199254740992.0) * 4.0 - 2.0);
    }
}
}  // namespace

int fesomc_closure_time(fesomc_closure *c, int64_t n, int32_t reps, int32_t bf16, double *ms) {
    if (!c || n < 1 || reps < 1 || !ms) return FESOMC_EINVAL;
    LcNet *net = c->net;
    if (bf16 && !lc_tc_supported(net)) return FESOMC_EINVAL;
    if (bf16 && !net->tc_ready) {
        int rc = lc_tc_prepare(net);
        if (rc) return rc;
    }
    float *dx = nullptr, *dy = nullptr, *ba = nullptr, *bb = nullptr;
    int rc = FESOMC_OK;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaMalloc(&dx, sizeof(float) * n * net->IN) || cudaMalloc(&dy, sizeof(float) * n * net->OUT) ||
        (!bf16 && (cudaMalloc(&ba, sizeof(float) * n * kLcHidden) || cudaMalloc(&bb, sizeof(float) * n * kLcHidden))))
        rc = FESOMC_ENOMEM;
    if (!rc && (cudaEventCreate(&e0) || cudaEventCreate(&e1))) rc = FESOMC_ECUDA;
    if (!rc) {
        k_lc_fill<<<grid_for(n * net->IN, 256), 256>>>(n * net->IN, dx, 12345ULL);
        auto once = [&]() {
            return bf16 ? lc_forward_tc(net, dx, n, dy, nullptr) : lc_forward_full(net, dx, n, dy, ba, bb, nullptr);
        };
        rc = once();   // warm-up
        if (!rc && cudaEventRecord(e0) != cudaSuccess) rc = FESOMC_ECUDA;
        for (int r = 0; r < reps && !rc; ++r) rc = once();
        if (!rc && (cudaEventRecord(e1) || cudaEventSynchronize(e1))) rc = FESOMC_ECUDA;
        float t = 0.0f;
        if (!rc && cudaEventElapsedTime(&t, e0, e1) != cudaSuccess) rc = FESOMC_ECUDA;
        *ms = t / reps;
        if (!rc && bf16) {
            unsigned int err = 0;
            if (cudaMemcpy(&err, net->tc_err, sizeof(err), cudaMemcpyDeviceToHost) != cudaSuccess || err) rc = FESOMC_ECUDA;
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(dx); cudaFree(dy); cudaFree(ba); cudaFree(bb);
    return rc;
}

int fesomc_closure_attach(fesomc_model *m, fesomc_closure *c, int32_t judge_every, int32_t bf16) {
    if (!m || judge_every < 0) return FESOMC_EINVAL;
    drop_graph(m);
    if (!c) {
        m->lc_on = false;
        m->lc = nullptr;
        return FESOMC_OK;
    }
    if (c->net->NS != m->d.NS || m->p.ver_mix != 3) return FESOMC_EINVAL;
    if (c->net->n_train < 1) return FESOMC_ESTATE;   // no statistics: fesomc_closure_fit first
    if (bf16 && !lc_tc_supported(c->net)) return FESOMC_EINVAL;
    int rc = lc_model_buffers(m, c);
    if (rc) return rc;
    if (bf16 && (rc = lc_tc_prepare(c->net))) return rc;
    if (!bf16 && (rc = lc_fp32_buffers(m))) return rc;
    m->lc_bf16 = bf16 != 0;
    m->lcv.rules = c->net->rules;
    CK(cudaMemset(m->lcv.acc, 0, 4 * sizeof(unsigned long long)));
    CK(cudaMemset(m->lcv.judge, 0, 3 * sizeof(double)));
    CK(cudaDeviceSynchronize());   // the fills (legacy stream) before the model stream's next step
    m->lc = c->net;
    m->lc_on = true;
    m->lc_judge_every = judge_every;
    m->lc_steps = 0;
    m->lc_judges = 0;
    return FESOMC_OK;
}

int fesomc_closure_set_rules(fesomc_closure *c, int32_t rules) {
    if (!c || (rules & ~(fesomc::kLcRuleUnstable | fesomc::kLcRuleBoundary))) return FESOMC_EINVAL;
    c->net->rules = rules;
    return FESOMC_OK;
}

int fesomc_closure_stats(fesomc_model *m, fesomc_closure_report *r) {
    if (!m || !r) return FESOMC_EINVAL;
    std::memset(r, 0, sizeof(*r));
    r->steps = m->lc_steps;
    r->judge_steps = m->lc_judges;
    if (!m->lcv.acc) return FESOMC_OK;
    unsigned long long acc[4];
    double j[3];
    CK(cudaStreamSynchronize(m->stream));
    CK(cudaMemcpy(acc, m->lcv.acc, sizeof(acc), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(j, m->lcv.judge, sizeof(j), cudaMemcpyDeviceToHost));
    r->wet_columns = (int64_t)acc[0];
    r->out_of_envelope = (int64_t)acc[1];
    r->dry_columns = (int64_t)acc[2];
    r->judge_values = (int64_t)j[1];
    r->judge_rms_log = j[1] > 0 ? std::sqrt(j[0] / j[1]) : 0.0;
    r->judge_max_log = j[2];
    return FESOMC_OK;
}

int fesomc_gpu_d3end_iterations(fesomc_model *m, int32_t nsteps, int32_t *iters) {
    if (!m || nsteps < 1 || !iters || m->p.ver_mix != 3) return FESOMC_EINVAL;
    int *buf = nullptr;
    int rc = dalloc(m, &buf, (size_t)m->d.N);
    if (rc) return rc;
    drop_graph(m);                   // the graph holds the kernels' parameters: capture again
    m->d.d3_iters = buf;
    m->d32.d3_iters = buf;
    rc = run_steps(m, nsteps);
    m->d.d3_iters = nullptr;
    m->d32.d3_iters = nullptr;
    drop_graph(m);
    if (rc) return rc;
    if ((rc = collect_status(m))) return rc;
    CK(cudaMemcpy(iters, buf, sizeof(int) * (size_t)m->d.N, cudaMemcpyDeviceToHost));
    return status_code(m->status_acc);
}

int fesomc_gpu_set_device(int32_t device) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return FESOMC_ECUDA;
    if (device < 0 || device >= n) return FESOMC_EINVAL;
    CK(cudaSetDevice(device));
    return FESOMC_OK;
}

const char *fesomc_gpu_version(void) { return "fesomc-b200 0.1 (sm_100a, FP64 plain path)"; }

int64_t fesomc_gpu_kernel_launches(fesomc_model *m) { return m ? m->launches : 0; }

}  // extern "C"
