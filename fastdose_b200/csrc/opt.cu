// opt.cu -- the IMRT fluence optimizer on the device.
//
// Objective (eval_g::evaluate, IMRTOpt/src/IMRTOptUtils.cu:74-156):
//   g(x) = 1/2 [ sum_PTV w_min min(Ax - d_min, 0)^2 + sum_VOI w_max max(Ax - d_max, 0)^2
//               + sum_OAR w_oar (Ax)^2 ]
//        + eta [ sum |p| + 1/(2 gamma) sum (p - Dx)^2 ],   p = sign(Dx) max(|Dx| - gamma, 0)
// Gradient (eval_grad::evaluate, IMRTOptUtils.cu:512-631):
//   A^T [w_min prox1 (+) w_oar Ax_OAR + w_max prox2] + (eta/gamma) D^T (Dx - p)
// Group prox (proxL2Onehalf_QL_gpu, IMRTOpt/src/IMRTOptimize_var1.cu:502-570)
// and the accelerated proximal-gradient loops BOO_IMRT_L2OneHalf_gpu_QL and
// polish_BOO_IMRT_gpu (IMRTOpt/src/IMRTOptimize.cu:16-194, 391-476).
//
// Layout: the four matrices are stream-SpMV CSR (spmv.cu); every vector is a
// flat FP32 array.  The elementwise terms are one fused pass over the VOI and
// D rows that also writes the gradient inputs; every sum (objective terms,
// group norms, line-search terms) accumulates in FP64 through fixed-shape
// two-stage reductions, so results do not depend on scheduling.  A line-search
// trial runs entirely on the device and returns its four scalars and the group
// norms in one pinned copy: one host synchronisation per trial, where the
// reference synchronises after nearly every kernel.
#include <algorithm>
#include <cmath>
#include <type_traits>
#include <vector>

#include <cub/block/block_reduce.cuh>

#include "opt_internal.cuh"

namespace fd2 {

namespace {

constexpr int kRedBlocks = 592;  // 4 per SM
constexpr int kRedThreads = 256;
constexpr int kTerms = 5;
constexpr float kEps = 1e-4f;  // eps_fastdose, FastDoseLib/include/macros.h:21

// slots of the reduced scalars
enum Slot { S_G = 0, S_GY = 1, S_GX = 2, S_DXY = 3, S_NXY = 4, S_TERMS = 8, S_COUNT = 16 };

template <int K>
__device__ __forceinline__ void block_partials(double (&v)[K], double* __restrict__ part) {
    typedef cub::BlockReduce<double, kRedThreads> R;
    __shared__ typename R::TempStorage tmp;
#pragma unroll
    for (int q = 0; q < K; q++) {
        const double s = R(tmp).Sum(v[q]);
        if (threadIdx.x == 0) part[(size_t)blockIdx.x * K + q] = s;
        __syncthreads();
    }
}

// Objective terms over the VOI rows (s1, s2, s3) and the D rows (s4, s5);
// optionally the gradient inputs g1 [nv] and g2 [m] (FP32, as the reference's
// d_calc_grad_term1_input / d_calc_grad_term2_input).
__global__ void __launch_bounds__(kRedThreads) objective_terms(
    const float* __restrict__ Ax, const float* __restrict__ Dx, int64_t n_ptv, int64_t nv, int64_t m,
    const float* __restrict__ max_dose, const float* __restrict__ max_w, const float* __restrict__ min_dose,
    const float* __restrict__ min_w, const float* __restrict__ oar_w, float gamma, float eta,
    float* __restrict__ g1, float* __restrict__ g2, double* __restrict__ part) {
    double s[kTerms] = {0, 0, 0, 0, 0};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nv; i += stride) {
        const float ax = Ax[i];
        const double d2 = (double)ax - (double)max_dose[i];
        const double dpr2 = d2 > 0 ? d2 : 0.0;  // d_calc_prox2
        s[1] += fabs((double)max_w[i] * dpr2 * dpr2);
        float v1;
        if (i < n_ptv) {
            const double d1 = (double)ax - (double)min_dose[i];
            const double dpr1 = d1 < 0 ? d1 : 0.0;  // d_calc_prox1
            s[0] += fabs((double)min_w[i] * dpr1 * dpr1);
            v1 = __fmul_rn(min_w[i], fminf(__fsub_rn(ax, min_dose[i]), 0.0f));
        } else {
            const float w = oar_w[i - n_ptv];
            s[2] += fabs((double)w * (double)ax * (double)ax);
            v1 = __fmul_rn(w, ax);
        }
        if (g1) g1[i] = __fadd_rn(v1, __fmul_rn(max_w[i], fmaxf(__fsub_rn(ax, max_dose[i]), 0.0f)));
    }
    const float eg = eta / gamma;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += stride) {
        const float t4 = Dx[i];
        const double dt = t4;
        double mm = fabs(dt) - (double)gamma;
        mm = mm > 0 ? mm : 0.0;
        const double dpr4 = mm * (double)((t4 > 0.0f) - (t4 < 0.0f));  // d_prox1Norm
        s[3] += fabs(dpr4);
        s[4] += (dpr4 - dt) * (dpr4 - dt);
        if (g2) {
            const float pr4 = __fmul_rn(fmaxf(__fsub_rn(fabsf(t4), gamma), 0.0f), (float)((t4 > 0.0f) - (t4 < 0.0f)));
            g2[i] = __fmul_rn(__fsub_rn(t4, pr4), eg);
        }
    }
    block_partials<kTerms>(s, part);
}

// Sums the per-block partials of K terms in block order.
template <int K>
__global__ void __launch_bounds__(kRedThreads) finish_sums(const double* __restrict__ part, int n_blocks,
                                                           double* __restrict__ out) {
    typedef cub::BlockReduce<double, kRedThreads> R;
    __shared__ typename R::TempStorage tmp;
    for (int q = 0; q < K; q++) {
        double s = 0;
        for (int b = threadIdx.x; b < n_blocks; b += kRedThreads) s += part[(size_t)b * K + q];
        s = R(tmp).Sum(s);
        if (threadIdx.x == 0) out[q] = s;
        __syncthreads();
    }
}

// objective value from the five terms into out[slot]
__global__ void objective_value(const double* __restrict__ terms, float gamma, float eta, double* __restrict__ out,
                                int slot) {
    if (threadIdx.x == 0 && blockIdx.x == 0)
        out[slot] = 0.5 * (terms[0] + terms[1] + terms[2]) +
                    (double)eta * (terms[3] + 0.5 / (double)gamma * terms[4]);
}

__global__ void add_vectors(const float* __restrict__ a, const float* __restrict__ b, float* __restrict__ out,
                            int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = __fadd_rn(a[i], b[i]);  // d_elementWiseAdd
}

// y = (1 - theta) x + theta v when step[2] != 0, else y = x; theta = step[0]
// (the trial's scalars come from device memory, so one captured graph serves
// every trial)
__global__ void extrapolate(const float* __restrict__ x, const float* __restrict__ v, const float* __restrict__ step,
                            float* __restrict__ y, int64_t n) {
    const float theta = step[0], a = 1.0f - theta;
    const bool ex = step[2] != 0.0f;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] = ex ? __fadd_rn(__fmul_rn(a, x[i]), __fmul_rn(theta, v[i])) : x[i];
}

// v = (1/theta) x + (1 - 1/theta) xkm1 ; xkm1 = x
__global__ void momentum(const float* __restrict__ x, float iot, float* __restrict__ xkm1, float* __restrict__ v,
                         int64_t n) {
    const float b = 1.0f - iot;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float xi = x[i];
        v[i] = __fadd_rn(__fmul_rn(iot, xi), __fmul_rn(b, xkm1[i]));
        xkm1[i] = xi;
    }
}

// x = max(y - t g, 0)   (the polish projection), t = *t_dev
__global__ void project_step(const float* __restrict__ y, const float* __restrict__ g, const float* __restrict__ t_dev,
                             float* __restrict__ x, int64_t n) {
    const float t = *t_dev;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] = fmaxf(__fadd_rn(y[i], __fmul_rn(-t, g[i])), 0.0f);
}

// d_proxL2Onehalf_calc_tHat (IMRTOptimize_var1.cu:544-570) in FP32, the
// reference's precision, with its zero-norm guard: the scale that minimises
// tau ||s g||^(1/2) + ||s g - g||^2 / 2 (closed form of the half-norm prox).
__device__ __forceinline__ float t_hat(float nrm2, float tau) {
    float n34 = 1008611.0f;
    if (nrm2 > kEps) n34 = powf(nrm2, -0.75f);
    const float alpha = tau * n34;
    if (alpha > 0.5443310539518174f) return 0.0f;  // 2 sqrt(6) / 9
    float s = acosf(alpha * 1.299038105676658f);  // 3 sqrt(3) / 4
    s = sinf((s + 1.5707963267948966f) / 3.0f) * 1.1547005383792517f;  // 2 / sqrt(3)
    return s * s;
}

// One block per group: in = max(y - t g, 0) (or y itself when g is null),
// prox = tHat(||in||^2, tau) in, nrm = ||prox||, with FP64 norm sums.
// tau = tau[r] when given, else w[r] * t; t = *t_dev when t_dev is given.
__global__ void __launch_bounds__(kRedThreads) group_prox(const int64_t* __restrict__ go, const float* __restrict__ y,
                                                          const float* __restrict__ g, float t,
                                                          const float* __restrict__ t_dev,
                                                          const float* __restrict__ w, const float* __restrict__ tau,
                                                          float* __restrict__ x, float* __restrict__ nrm) {
    if (t_dev) t = *t_dev;
    typedef cub::BlockReduce<double, kRedThreads> R;
    __shared__ typename R::TempStorage tmp;
    __shared__ float s_th;
    const int64_t r = blockIdx.x, a = go[r], b = go[r + 1];
    double n2 = 0;
    for (int64_t i = a + threadIdx.x; i < b; i += kRedThreads) {
        const float in = g ? fmaxf(__fadd_rn(y[i], __fmul_rn(-t, g[i])), 0.0f) : y[i];
        n2 += (double)in * in;
    }
    n2 = R(tmp).Sum(n2);
    if (threadIdx.x == 0) s_th = t_hat((float)n2, tau ? tau[r] : __fmul_rn(w[r], t));
    __syncthreads();
    const float th = s_th;
    double m2 = 0;
    for (int64_t i = a + threadIdx.x; i < b; i += kRedThreads) {
        const float in = g ? fmaxf(__fadd_rn(y[i], __fmul_rn(-t, g[i])), 0.0f) : y[i];
        const float p = __fmul_rn(th, in);
        x[i] = p;
        m2 += (double)p * p;
    }
    m2 = R(tmp).Sum(m2);
    if (threadIdx.x == 0) nrm[r] = sqrtf((float)m2);
}

// line-search terms: sum g (x - y), sum (x - y)^2
__global__ void __launch_bounds__(kRedThreads) step_terms(const float* __restrict__ g, const float* __restrict__ x,
                                                          const float* __restrict__ y, int64_t n,
                                                          double* __restrict__ part) {
    double s[2] = {0, 0};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float d = __fsub_rn(x[i], y[i]);
        s[0] += (double)g[i] * d;
        s[1] += (double)d * d;
    }
    block_partials<2>(s, part);
}

template <typename T>
__device__ __forceinline__ float as_float(T v) {
    if constexpr (std::is_same<T, float>::value) return v;
    else if constexpr (std::is_same<T, __half>::value) return __half2float(v);
    else return __bfloat162float(v);
}

// per beamlet: the sum of its PTV-row entries (AT rows list VOI columns
// ascending, PTV first), scale applied
template <typename T>
__global__ void ptv_column_sums(const int64_t* __restrict__ off, ColView col,
                                const T* __restrict__ val, const float* __restrict__ row_scale, int64_t rows,
                                int64_t n_ptv, double* __restrict__ out) {
    const int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= rows) return;
    double s = 0;
    for (int64_t k = off[r] + lane; k < off[r + 1]; k += 32) {
        if (col.at(k) >= n_ptv) break;
        s += (double)as_float(val[slot(k)]);
    }
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) out[r] = s * (row_scale ? (double)row_scale[r] : 1.0);
}

unsigned vec_blocks(int64_t n) { return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 8)); }

}  // namespace
}  // namespace fd2

struct fd2_opt_problem {
    fd2_context* ctx = nullptr;
    const fd2_matrix *A = nullptr, *AT = nullptr, *D = nullptr, *DT = nullptr;
    int64_t n_ptv = 0, n_oar = 0, nv = 0, n = 0, m = 0;
    float gamma = 1.0f, eta = 0.1f;
    float *d_max_dose = nullptr, *d_max_w = nullptr, *d_min_dose = nullptr, *d_min_w = nullptr, *d_oar_w = nullptr;
    float *d_Ax = nullptr, *d_Dx = nullptr, *d_g1 = nullptr, *d_g2 = nullptr, *d_o1 = nullptr, *d_o2 = nullptr;
    float *d_y = nullptr, *d_g = nullptr, *d_x = nullptr;
    double *d_part = nullptr, *d_red = nullptr;
    double* h_red = nullptr;  // pinned [S_COUNT]
    // the trial's scalars (theta, t, extrapolated) in pinned host memory and
    // on the device, and the trial captured as a CUDA graph
    float* h_step = nullptr;  // pinned [4]
    float* d_step = nullptr;  // [4]
    bool use_graph = true;
    // row-sharded problems: the caller's sum over ranks of a device FP64 buffer
    fd2_reduce_fn reducer = nullptr;
    void* reducer_user = nullptr;
    double* d_rbuf = nullptr;  // [n + 3]
    cudaGraphExec_t trial_exec = nullptr;
    const float *graph_xkm1 = nullptr, *graph_vkm1 = nullptr;
    int64_t graph_groups = -1;
    uint64_t graph_kernels = 0;
    // group buffers (BOO)
    int64_t groups_cap = 0;
    int64_t* d_go = nullptr;
    float *d_w = nullptr, *d_nrm = nullptr;
    float* h_nrm = nullptr;  // pinned [groups_cap]
    std::vector<void*> owned;
};

namespace fd2 {
namespace {

int palloc(fd2_opt_problem* p, void** ptr, size_t bytes) {
    FD2_CHECK_CUDA(cudaMalloc(ptr, std::max<size_t>(bytes, 16)));
    p->owned.push_back(*ptr);
    return FD2_OK;
}

// Row-sharded problems: buf = [the three VOI-row terms, the partial A^T g1]
// in FP64, summed over the ranks by the caller's reducer, and unpacked.  The
// fluence-gradient terms and D^T g2 are the same on every rank and stay local.
__global__ void pack_partials(const double* __restrict__ terms, const float* __restrict__ o1, int64_t n,
                              double* __restrict__ buf) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n + 3; i += stride)
        buf[i] = i < 3 ? terms[i] : (double)o1[i - 3];
}
__global__ void unpack_partials(const double* __restrict__ buf, int64_t n, double* __restrict__ terms,
                                float* __restrict__ o1) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n + 3; i += stride) {
        if (i < 3)
            terms[i] = buf[i];
        else
            o1[i - 3] = (float)buf[i];
    }
}

int reduce_partials(fd2_opt_problem* p, bool with_grad) {
    cudaStream_t st = p->ctx->stream;
    const int64_t n = with_grad ? p->n : 0;
    pack_partials<<<vec_blocks(n + 3), 256, 0, st>>>(p->d_red + S_TERMS, p->d_o1, n, p->d_rbuf);
    FD2_CHECK_CUDA(cudaGetLastError());
    FD2_CHECK_CUDA(cudaStreamSynchronize(st));  // the reducer works on its own stream
    const int rc = p->reducer(p->reducer_user, p->d_rbuf, n + 3, st);
    FD2_REQUIRE(rc == 0, FD2_ERR_CUDA, "optimizer: the rank reduction failed (%d)", rc);
    unpack_partials<<<vec_blocks(n + 3), 256, 0, st>>>(p->d_rbuf, n, p->d_red + S_TERMS, p->d_o1);
    FD2_CHECK_CUDA(cudaGetLastError());
    p->ctx->launches += 2;
    return FD2_OK;
}

// objective of x into d_red[slot]; with grad: the gradient into grad
int objective(fd2_opt_problem* p, const float* x, float* grad, int slot) {
    cudaStream_t st = p->ctx->stream;
    FD2_TRY(matrix_spmv(p->A, x, p->d_Ax, st));
    if (p->m) FD2_TRY(matrix_spmv(p->D, x, p->d_Dx, st));
    objective_terms<<<kRedBlocks, kRedThreads, 0, st>>>(p->d_Ax, p->d_Dx, p->n_ptv, p->nv, p->m, p->d_max_dose,
                                                        p->d_max_w, p->d_min_dose, p->d_min_w, p->d_oar_w, p->gamma,
                                                        p->eta, grad ? p->d_g1 : nullptr, grad ? p->d_g2 : nullptr,
                                                        p->d_part);
    finish_sums<kTerms><<<1, kRedThreads, 0, st>>>(p->d_part, kRedBlocks, p->d_red + S_TERMS);
    FD2_CHECK_CUDA(cudaGetLastError());
    p->ctx->launches += 2;
    if (grad) {
        if (p->m) {
            FD2_TRY(matrix_spmv(p->DT, p->d_g2, p->d_o2, st));
        } else {
            FD2_CHECK_CUDA(cudaMemsetAsync(p->d_o2, 0, p->n * sizeof(float), st));
        }
        FD2_TRY(matrix_spmv(p->AT, p->d_g1, p->d_o1, st));
    }
    if (p->reducer) FD2_TRY(reduce_partials(p, grad != nullptr));
    objective_value<<<1, 32, 0, st>>>(p->d_red + S_TERMS, p->gamma, p->eta, p->d_red, slot);
    p->ctx->launches += 1;
    if (grad) {
        add_vectors<<<vec_blocks(p->n), 256, 0, st>>>(p->d_o1, p->d_o2, grad, p->n);
        p->ctx->launches += 1;
    }
    FD2_CHECK_CUDA(cudaGetLastError());
    return FD2_OK;
}

int read_scalars(fd2_opt_problem* p, int64_t n_groups) {
    cudaStream_t st = p->ctx->stream;
    FD2_CHECK_CUDA(cudaMemcpyAsync(p->h_red, p->d_red, S_COUNT * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (n_groups > 0)
        FD2_CHECK_CUDA(cudaMemcpyAsync(p->h_nrm, p->d_nrm, n_groups * sizeof(float), cudaMemcpyDeviceToHost, st));
    FD2_CHECK_CUDA(cudaStreamSynchronize(st));
    return FD2_OK;
}

void drop_graph(fd2_opt_problem* p);

int ensure_groups(fd2_opt_problem* p, int64_t n_groups) {
    if (n_groups <= p->groups_cap) return FD2_OK;
    drop_graph(p);  // its copies name the group buffers being replaced
    FD2_TRY(palloc(p, (void**)&p->d_go, (n_groups + 1) * sizeof(int64_t)));
    FD2_TRY(palloc(p, (void**)&p->d_w, n_groups * sizeof(float)));
    FD2_TRY(palloc(p, (void**)&p->d_nrm, n_groups * sizeof(float)));
    if (p->h_nrm) cudaFreeHost(p->h_nrm);
    p->h_nrm = nullptr;
    FD2_CHECK_CUDA(cudaMallocHost(&p->h_nrm, n_groups * sizeof(float)));
    p->groups_cap = n_groups;
    return FD2_OK;
}

// One line-search trial at step t: y from (theta, xkm1, vkm1); x = prox or
// projection of y - t grad g(y); leaves gx, gy, <grad, x - y>, ||x - y||^2 in h_red.
// The work of one trial, enqueued on the context's stream without a host
// wait: the scalars' upload, the products and reductions, the read-back of
// the four scalars and the group norms into pinned memory.
int trial_enqueue(fd2_opt_problem* p, const fd2_opt_state_t* st, int64_t n_groups) {
    cudaStream_t s = p->ctx->stream;
    const int64_t n = p->n;
    FD2_CHECK_CUDA(cudaMemcpyAsync(p->d_step, p->h_step, 4 * sizeof(float), cudaMemcpyHostToDevice, s));
    extrapolate<<<vec_blocks(n), 256, 0, s>>>(st->d_xkm1, st->d_vkm1, p->d_step, p->d_y, n);
    FD2_TRY(objective(p, p->d_y, p->d_g, S_GY));
    if (n_groups > 0)
        group_prox<<<(unsigned)n_groups, kRedThreads, 0, s>>>(p->d_go, p->d_y, p->d_g, 0.0f, p->d_step + 1, p->d_w,
                                                              nullptr, p->d_x, p->d_nrm);
    else
        project_step<<<vec_blocks(n), 256, 0, s>>>(p->d_y, p->d_g, p->d_step + 1, p->d_x, n);
    FD2_TRY(objective(p, p->d_x, nullptr, S_GX));
    step_terms<<<kRedBlocks, kRedThreads, 0, s>>>(p->d_g, p->d_x, p->d_y, n, p->d_part);
    finish_sums<2><<<1, kRedThreads, 0, s>>>(p->d_part, kRedBlocks, p->d_red + S_DXY);
    FD2_CHECK_CUDA(cudaGetLastError());
    p->ctx->launches += 5;
    FD2_CHECK_CUDA(cudaMemcpyAsync(p->h_red, p->d_red, S_COUNT * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (n_groups > 0)
        FD2_CHECK_CUDA(cudaMemcpyAsync(p->h_nrm, p->d_nrm, n_groups * sizeof(float), cudaMemcpyDeviceToHost, s));
    return FD2_OK;
}

void drop_graph(fd2_opt_problem* p) {
    if (p->trial_exec) cudaGraphExecDestroy(p->trial_exec);
    p->trial_exec = nullptr;
    p->graph_groups = -1;
}

// The trial's launches as one CUDA graph, captured for this state's vectors and
// group count; replays read the scalars from p->h_step at execution.
int capture_trial(fd2_opt_problem* p, const fd2_opt_state_t* st, int64_t n_groups) {
    drop_graph(p);
    cudaStream_t s = p->ctx->stream;
    const uint64_t before = p->ctx->launches;
    FD2_CHECK_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    const int rc = trial_enqueue(p, st, n_groups);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(s, &graph);
    if (rc || e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        if (!rc) FD2_CHECK_CUDA(e);
        return rc;
    }
    const cudaError_t ei = cudaGraphInstantiate(&p->trial_exec, graph, 0);
    cudaGraphDestroy(graph);
    FD2_CHECK_CUDA(ei);
    p->graph_xkm1 = st->d_xkm1;
    p->graph_vkm1 = st->d_vkm1;
    p->graph_groups = n_groups;
    p->graph_kernels = p->ctx->launches - before;
    p->ctx->launches = before;
    return FD2_OK;
}

int trial(fd2_opt_problem* p, const fd2_opt_state_t* st, float theta, bool extrapolated, float t, int64_t n_groups) {
    cudaStream_t s = p->ctx->stream;
    p->h_step[0] = theta;
    p->h_step[1] = t;
    p->h_step[2] = extrapolated ? 1.0f : 0.0f;
    if (p->use_graph) {
        if (!p->trial_exec || p->graph_xkm1 != st->d_xkm1 || p->graph_vkm1 != st->d_vkm1 ||
            p->graph_groups != n_groups)
            FD2_TRY(capture_trial(p, st, n_groups));
        FD2_CHECK_CUDA(cudaGraphLaunch(p->trial_exec, s));
        p->ctx->launches += p->graph_kernels;
    } else {
        FD2_TRY(trial_enqueue(p, st, n_groups));
    }
    FD2_CHECK_CUDA(cudaStreamSynchronize(s));
    return FD2_OK;
}

// theta of the accelerated step (IMRTOptimize.cu:78-84): the positive root of
// tkm1 theta^2 + t theta_km1^2 theta - t theta_km1^2 = 0
float next_theta(float tkm1, float t, float theta_km1) {
    const float aa = tkm1, bb = t * theta_km1 * theta_km1, cc = -bb;
    return (-bb + sqrtf(bb * bb - 4 * aa * cc)) / (2 * aa);
}

constexpr int kMaxHalvings = 200;  // a step below 2^-200 t means the line search cannot succeed

int solve(fd2_opt_problem* p, int64_t n_groups, const int64_t* h_go, float* h_w, int change_trigger, int iters_global,
          int iters_local, int want, fd2_opt_state_t* st) {
    cudaStream_t s = p->ctx->stream;
    const int64_t n = p->n;
    if (n_groups > 0) {
        FD2_TRY(ensure_groups(p, n_groups));
        FD2_CHECK_CUDA(cudaMemcpyAsync(p->d_go, h_go, (n_groups + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, s));
        FD2_CHECK_CUDA(cudaMemcpyAsync(p->d_w, h_w, n_groups * sizeof(float), cudaMemcpyHostToDevice, s));
        st->stop = 0;
    }
    float t = st->tkm1, theta = 1.0f;
    st->trials = 0;
    int k_local = 0;
    for (; st->k_global < iters_global && k_local < iters_local; st->k_global++, k_local++) {
        if (st->k_global < 50 || st->k_global % 5 == 0) t /= 0.5f;
        double gx = 0;
        for (int halvings = 0;; halvings++) {
            FD2_REQUIRE(halvings < kMaxHalvings, FD2_ERR_WATCHDOG,
                        "optimizer: no accepted step after %d halvings (t=%g)", kMaxHalvings, (double)t);
            st->trials++;
            const bool ex = st->k_global > 1;
            theta = ex ? next_theta(st->tkm1, t, st->theta_km1) : 1.0f;
            FD2_TRY(trial(p, st, theta, ex, t, n_groups));
            gx = p->h_red[S_GX];
            const double rhs = p->h_red[S_GY] + p->h_red[S_DXY] + (0.5 / (double)t) * p->h_red[S_NXY];
            if (gx <= rhs) break;
            t *= 0.5f;
        }
        const float iot = 1.0f / theta;
        momentum<<<vec_blocks(n), 256, 0, s>>>(p->d_x, iot, st->d_xkm1, st->d_vkm1, n);
        FD2_CHECK_CUDA(cudaGetLastError());
        p->ctx->launches += 1;
        st->theta_km1 = theta;
        st->tkm1 = t;
        if (n_groups > 0) {
            double cost = 0;
            float active = 0;
            for (int64_t r = 0; r < n_groups; r++) {
                cost += (double)h_w[r] * std::sqrt((double)p->h_nrm[r]);
                active += p->h_nrm[r] > kEps;
            }
            if (st->h_loss) st->h_loss[st->k_global] = (float)(cost + gx);
            if (st->h_nrm) std::copy(p->h_nrm, p->h_nrm + n_groups, st->h_nrm);
            st->num_active = active;
            if (active - kEps <= want) {
                st->stop = 1;
                break;
            }
            if ((st->k_global + 1) % change_trigger == 0) {  // adaptive beam weights (IMRTOptimize.cu:160-181)
                float sc = 1.0f;
                if (active >= 2 * want) sc = 2.0f;
                else if (active >= 1.5f * want) sc = 1.5f;
                else if (active >= 1.05f * want) sc = 1.2f;
                else if (active < want) sc = 0.3333f;
                if (sc != 1.0f) {
                    for (int64_t r = 0; r < n_groups; r++) h_w[r] *= sc;
                    FD2_CHECK_CUDA(cudaMemcpyAsync(p->d_w, h_w, n_groups * sizeof(float), cudaMemcpyHostToDevice, s));
                }
            }
        } else if (st->h_loss) {
            st->h_loss[st->k_global] = (float)gx;
        }
    }
    if (n_groups > 0 && st->k_global == iters_global) st->stop = 1;
    FD2_CHECK_CUDA(cudaStreamSynchronize(s));
    return FD2_OK;
}

}  // namespace
}  // namespace fd2

using namespace fd2;

extern "C" {

int fd2_opt_problem_create(fd2_context* ctx, const fd2_matrix* A, const fd2_matrix* AT, const fd2_matrix* D,
                           const fd2_matrix* DT, int64_t n_ptv, int64_t n_oar, const float* h_max_dose,
                           const float* h_max_weights, const float* h_min_dose, const float* h_min_weights,
                           const float* h_oar_weights, float gamma, float eta, fd2_opt_problem** out) {
    FD2_REQUIRE(ctx && A && AT && D && DT && out && h_max_dose && h_max_weights &&
                    (n_ptv == 0 || (h_min_dose && h_min_weights)) && (n_oar == 0 || h_oar_weights),
                FD2_ERR_INVALID_ARGUMENT, "opt_problem_create: null argument");
    const int64_t nv = n_ptv + n_oar;
    FD2_REQUIRE(n_ptv >= 0 && n_oar >= 0 && A->rows == nv && AT->cols == nv && AT->rows == A->cols &&
                    D->cols == A->cols && DT->rows == D->cols && DT->cols == D->rows,
                FD2_ERR_INVALID_ARGUMENT,
                "opt_problem_create: shapes A %lldx%lld AT %lldx%lld D %lldx%lld DT %lldx%lld for %lld+%lld VOI rows",
                (long long)A->rows, (long long)A->cols, (long long)AT->rows, (long long)AT->cols, (long long)D->rows,
                (long long)D->cols, (long long)DT->rows, (long long)DT->cols, (long long)n_ptv, (long long)n_oar);
    FD2_REQUIRE(gamma > 0.0f, FD2_ERR_INVALID_ARGUMENT, "opt_problem_create: gamma must be positive");
    auto* p = new fd2_opt_problem();
    p->ctx = ctx;
    p->A = A;
    p->AT = AT;
    p->D = D;
    p->DT = DT;
    p->n_ptv = n_ptv;
    p->n_oar = n_oar;
    p->nv = nv;
    p->n = A->cols;
    p->m = D->rows;
    p->gamma = gamma;
    p->eta = eta;
    cudaStream_t st = ctx->stream;
    int rc = FD2_OK;
    auto up = [&](float** d, const float* h, int64_t n) {
        if (rc) return;
        rc = palloc(p, (void**)d, n * sizeof(float));
        if (!rc && n && cudaMemcpyAsync(*d, h, n * sizeof(float), cudaMemcpyHostToDevice, st) != cudaSuccess)
            rc = FD2_ERR_CUDA;
    };
    up(&p->d_max_dose, h_max_dose, nv);
    up(&p->d_max_w, h_max_weights, nv);
    up(&p->d_min_dose, h_min_dose, n_ptv);
    up(&p->d_min_w, h_min_weights, n_ptv);
    up(&p->d_oar_w, h_oar_weights, n_oar);
    const std::pair<float**, int64_t> bufs[] = {{&p->d_Ax, nv},  {&p->d_g1, nv}, {&p->d_Dx, p->m},
                                                {&p->d_g2, p->m}, {&p->d_o1, p->n}, {&p->d_o2, p->n},
                                                {&p->d_y, p->n},  {&p->d_g, p->n},  {&p->d_x, p->n}};
    for (const auto& q : bufs)
        if (!rc) rc = palloc(p, (void**)q.first, q.second * sizeof(float));
    if (!rc) rc = palloc(p, (void**)&p->d_part, (size_t)kRedBlocks * kTerms * sizeof(double));
    if (!rc) rc = palloc(p, (void**)&p->d_red, S_COUNT * sizeof(double));
    if (!rc && cudaMallocHost(&p->h_red, S_COUNT * sizeof(double)) != cudaSuccess) rc = FD2_ERR_OUT_OF_MEMORY;
    if (!rc && cudaMallocHost(&p->h_step, 4 * sizeof(float)) != cudaSuccess) rc = FD2_ERR_OUT_OF_MEMORY;
    if (!rc) rc = palloc(p, (void**)&p->d_step, 4 * sizeof(float));
    if (!rc && cudaMemsetAsync(p->d_red, 0, S_COUNT * sizeof(double), st) != cudaSuccess) rc = FD2_ERR_CUDA;
    if (!rc && cudaStreamSynchronize(st) != cudaSuccess) rc = FD2_ERR_CUDA;
    if (rc) {
        fd2_opt_problem_destroy(p);
        return rc;
    }
    *out = p;
    return FD2_OK;
}

int fd2_opt_problem_destroy(fd2_opt_problem* p) {
    if (!p) return FD2_OK;
    drop_graph(p);
    for (void* q : p->owned) cudaFree(q);
    if (p->h_red) cudaFreeHost(p->h_red);
    if (p->h_step) cudaFreeHost(p->h_step);
    if (p->h_nrm) cudaFreeHost(p->h_nrm);
    delete p;
    return FD2_OK;
}

int fd2_opt_problem_set_graph(fd2_opt_problem* p, int on) {
    FD2_REQUIRE(p, FD2_ERR_INVALID_ARGUMENT, "opt_problem_set_graph: null problem");
    p->use_graph = on != 0 && !p->reducer;
    if (!p->use_graph) drop_graph(p);
    return FD2_OK;
}

int fd2_opt_problem_set_reducer(fd2_opt_problem* p, fd2_reduce_fn fn, void* user) {
    FD2_REQUIRE(p, FD2_ERR_INVALID_ARGUMENT, "opt_problem_set_reducer: null problem");
    p->reducer = fn;
    p->reducer_user = user;
    if (fn) {
        p->use_graph = false;  // the reduction is a host call between kernels
        drop_graph(p);
        if (!p->d_rbuf) FD2_TRY(palloc(p, (void**)&p->d_rbuf, (p->n + 3) * sizeof(double)));
    }
    return FD2_OK;
}

int fd2_eval_g(fd2_opt_problem* p, const float* d_x, double* h_value) {
    FD2_REQUIRE(p && d_x && h_value, FD2_ERR_INVALID_ARGUMENT, "eval_g: null argument");
    FD2_TRY(objective(p, d_x, nullptr, S_G));
    FD2_TRY(read_scalars(p, 0));
    *h_value = p->h_red[S_G];
    return FD2_OK;
}

int fd2_eval_grad(fd2_opt_problem* p, const float* d_x, float* d_grad, double* h_value) {
    FD2_REQUIRE(p && d_x && d_grad && h_value, FD2_ERR_INVALID_ARGUMENT, "eval_grad: null argument");
    FD2_TRY(objective(p, d_x, d_grad, S_G));
    FD2_TRY(read_scalars(p, 0));
    *h_value = p->h_red[S_G];
    return FD2_OK;
}

int fd2_prox_l2onehalf(fd2_context* ctx, int64_t n_groups, const int64_t* d_go, const float* d_g0, const float* d_tau,
                       float* d_prox, float* d_nrm, void* stream) {
    FD2_REQUIRE(ctx && d_go && d_g0 && d_tau && d_prox && d_nrm, FD2_ERR_INVALID_ARGUMENT,
                "prox_l2onehalf: null argument");
    if (n_groups <= 0) return FD2_OK;
    group_prox<<<(unsigned)n_groups, kRedThreads, 0, (cudaStream_t)stream>>>(d_go, d_g0, nullptr, 0.0f, nullptr,
                                                                             nullptr, d_tau, d_prox, d_nrm);
    FD2_CHECK_CUDA(cudaGetLastError());
    ctx->launches += 1;
    return FD2_OK;
}

int fd2_beam_weights_init(fd2_opt_problem* p, int64_t n_groups, const int64_t* h_go, float* h_w) {
    FD2_REQUIRE(p && h_go && h_w && n_groups > 0, FD2_ERR_INVALID_ARGUMENT, "beam_weights_init: bad argument");
    FD2_REQUIRE(h_go[0] == 0 && h_go[n_groups] == p->n, FD2_ERR_INVALID_ARGUMENT,
                "beam_weights_init: groups must cover the %lld beamlets", (long long)p->n);
    const fd2_matrix* at = p->AT;
    cudaStream_t st = p->ctx->stream;
    double* d_s = nullptr;  // [rows] PTV sums, then this problem's PTV row count (summed over ranks)
    FD2_CHECK_CUDA(cudaMalloc(&d_s, (at->rows + 1) * sizeof(double)));
    const float* rs = at->scale_axis == FD2_SCALE_ROWS ? at->d_scale : nullptr;
    const unsigned blocks = (unsigned)((at->rows * 32 + 255) / 256);
    if (at->rows) {
        switch (at->value_type) {
            case FD2_VALUES_F16:
                ptv_column_sums<__half><<<blocks, 256, 0, st>>>(at->d_off, at->cols_view(), (const __half*)at->d_val, rs,
                                                               at->rows, p->n_ptv, d_s);
                break;
            case FD2_VALUES_BF16:
                ptv_column_sums<__nv_bfloat16><<<blocks, 256, 0, st>>>(
                    at->d_off, at->cols_view(), (const __nv_bfloat16*)at->d_val, rs, at->rows, p->n_ptv, d_s);
                break;
            default:
                ptv_column_sums<float><<<blocks, 256, 0, st>>>(at->d_off, at->cols_view(), (const float*)at->d_val, rs,
                                                              at->rows, p->n_ptv, d_s);
        }
    }
    std::vector<double> s(at->rows + 1);
    s[at->rows] = (double)p->n_ptv;
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_s + at->rows, &s[at->rows], sizeof(double), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && p->reducer) {  // the PTV rows are spread over the ranks
        e = cudaStreamSynchronize(st);
        if (e == cudaSuccess && p->reducer(p->reducer_user, d_s, at->rows + 1, st) != 0) {
            cudaFree(d_s);
            set_error("beam_weights_init: the rank reduction failed");
            return FD2_ERR_CUDA;
        }
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(s.data(), d_s, (at->rows + 1) * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(d_s);
    FD2_CHECK_CUDA(e);
    const double n_ptv = s[at->rows];  // all ranks' PTV rows
    FD2_REQUIRE(n_ptv > 0, FD2_ERR_INVALID_ARGUMENT, "beam_weights_init: no PTV rows");
    // w_b = sqrt(sum_PTV A_b 1 / (n_ptv nbl_b)), normalised to the max, floored at 0.1
    float mx = 0.0f;
    for (int64_t b = 0; b < n_groups; b++) {
        double acc = 0;
        for (int64_t j = h_go[b]; j < h_go[b + 1]; j++) acc += s[j];
        const int64_t nb = h_go[b + 1] - h_go[b];
        h_w[b] = std::sqrt((float)acc / (float)((int64_t)n_ptv * nb));
        mx = std::max(mx, h_w[b]);
    }
    for (int64_t b = 0; b < n_groups; b++) {
        h_w[b] /= mx;
        if (h_w[b] < 0.1f) h_w[b] = 0.1f;
    }
    return FD2_OK;
}

int fd2_boo_l2onehalf(fd2_opt_problem* p, int64_t n_groups, const int64_t* h_go, float* h_w, int show_trigger,
                      int change_weights_trigger, int iters_global, const int32_t* h_prune, int n_prune, int want,
                      fd2_opt_state_t* st) {
    FD2_REQUIRE(p && h_go && h_w && st && st->d_xkm1 && st->d_vkm1 && n_groups > 0 && change_weights_trigger > 0,
                FD2_ERR_INVALID_ARGUMENT, "boo_l2onehalf: bad argument");
    FD2_REQUIRE(h_go[0] == 0 && h_go[n_groups] == p->n, FD2_ERR_INVALID_ARGUMENT,
                "boo_l2onehalf: groups must cover the %lld beamlets", (long long)p->n);
    FD2_REQUIRE(st->tkm1 > 0.0f, FD2_ERR_INVALID_ARGUMENT, "boo_l2onehalf: step size must be positive");
    (void)show_trigger;  // the reference prints progress every show_trigger iterations
    int iters_local = iters_global;
    for (int i = 0; i < n_prune; i++)
        if (h_prune[i] > st->k_global) {
            iters_local = h_prune[i] - st->k_global;
            break;
        }
    return solve(p, n_groups, h_go, h_w, change_weights_trigger, iters_global, iters_local, want, st);
}

int fd2_polish(fd2_opt_problem* p, int iters_global, int iters_local, fd2_opt_state_t* st) {
    FD2_REQUIRE(p && st && st->d_xkm1 && st->d_vkm1, FD2_ERR_INVALID_ARGUMENT, "polish: bad argument");
    FD2_REQUIRE(st->tkm1 > 0.0f, FD2_ERR_INVALID_ARGUMENT, "polish: step size must be positive");
    return solve(p, 0, nullptr, nullptr, 1, iters_global, iters_local, 0, st);
}

int fd2_beam_orientation_optimization(fd2_context* ctx, const fd2_matrix* AT, const fd2_matrix* D, int64_t n_beams,
                                      const int64_t* h_beam_rows, const int64_t* h_d_rows, int64_t n_ptv,
                                      int64_t n_oar, const float* h_max_dose, const float* h_max_weights,
                                      const float* h_min_dose, const float* h_min_weights,
                                      const float* h_oar_weights, const fd2_boo_params_t* prm, const float* d_x0,
                                      float* h_costs, int32_t* h_active, float* h_norms, float* d_x,
                                      fd2_boo_result_t* result) {
    FD2_REQUIRE(ctx && AT && D && h_beam_rows && h_d_rows && prm && d_x0 && h_costs && h_active && h_norms && d_x &&
                    result && n_beams > 0,
                FD2_ERR_INVALID_ARGUMENT, "beam_orientation_optimization: bad argument");
    FD2_REQUIRE(h_beam_rows[0] == 0 && h_beam_rows[n_beams] == AT->rows && h_d_rows[0] == 0 &&
                    h_d_rows[n_beams] == D->rows && D->cols == AT->rows,
                FD2_ERR_INVALID_ARGUMENT, "beam_orientation_optimization: beam blocks do not match AT (%lld rows) and D "
                "(%lld x %lld)", (long long)AT->rows, (long long)D->rows, (long long)D->cols);
    FD2_REQUIRE(prm->step_size > 0.0f && prm->max_iter > 0 && prm->change_weights_trigger > 0,
                FD2_ERR_INVALID_ARGUMENT, "beam_orientation_optimization: bad parameters");
    cudaStream_t s = ctx->stream;
    const int64_t n_all = AT->rows;
    // x and v of the active beams, ping-ponged through the reductions
    float *xb[2] = {nullptr, nullptr}, *vb[2] = {nullptr, nullptr};
    auto release = [&]() {
        for (float* q : {xb[0], xb[1], vb[0], vb[1]})
            if (q) cudaFree(q);
    };
    for (float** q : {&xb[0], &xb[1], &vb[0], &vb[1]})
        if (cudaMalloc(q, std::max<int64_t>(n_all, 1) * sizeof(float)) != cudaSuccess) {
            release();
            set_error("beam_orientation_optimization: out of device memory");
            return FD2_ERR_OUT_OF_MEMORY;
        }
    int cur = 0;
    cudaError_t ce = cudaMemcpyAsync(xb[0], d_x0, n_all * sizeof(float), cudaMemcpyDeviceToDevice, s);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(vb[0], d_x0, n_all * sizeof(float), cudaMemcpyDeviceToDevice, s);
    if (ce != cudaSuccess) {
        release();
        FD2_CHECK_CUDA(ce);
    }
    std::vector<int64_t> active(n_beams);
    for (int64_t b = 0; b < n_beams; b++) active[b] = b;
    std::vector<float> w;  // weights of the active beams, in order
    fd2_opt_state_t st{};
    st.k_global = 0;
    st.theta_km1 = 0.0f;
    st.tkm1 = prm->step_size;
    *result = fd2_boo_result_t{};
    std::vector<float> nrm;
    int rc = FD2_OK;
    for (;;) {
        const int64_t na = (int64_t)active.size();
        bool identity = na == n_beams;
        for (int64_t j = 0; identity && j < na; j++) identity = active[j] == j;
        // the active beams' matrices: the inputs themselves while every beam is
        // active in its original order, else a selection
        fd2_matrix *ATs = nullptr, *As = nullptr, *Ds = nullptr, *DTs = nullptr;
        const fd2_matrix* ATp = AT;
        const fd2_matrix* Dp = D;
        if (!identity) {
            rc = matrix_select_blocks(AT, n_beams, h_beam_rows, nullptr, na, active.data(), &ATs);
            if (!rc) rc = matrix_select_blocks(D, n_beams, h_d_rows, h_beam_rows, na, active.data(), &Ds);
            ATp = ATs;
            Dp = Ds;
        }
        if (!rc) rc = matrix_transpose_fmt(ATp, ATp->index_format, &As);
        if (!rc) rc = matrix_transpose_fmt(Dp, Dp->index_format, &DTs);
        fd2_opt_problem* p = nullptr;
        if (!rc)
            rc = fd2_opt_problem_create(ctx, As, ATp, Dp, DTs, n_ptv, n_oar, h_max_dose, h_max_weights, h_min_dose,
                                        h_min_weights, h_oar_weights, prm->gamma, prm->eta, &p);
        std::vector<int64_t> go(na + 1, 0);
        for (int64_t j = 0; j < na; j++) go[j + 1] = go[j] + h_beam_rows[active[j] + 1] - h_beam_rows[active[j]];
        if (!rc && result->phases == 0) {  // beamWeightsInit_func over all beams, times beamWeight
            w.assign(na, 0.0f);
            rc = fd2_beam_weights_init(p, na, go.data(), w.data());
            for (float& q : w) q *= prm->beam_weight;
        }
        nrm.assign(na, 0.0f);
        if (!rc) {
            st.d_xkm1 = xb[cur];
            st.d_vkm1 = vb[cur];
            st.h_loss = h_costs;
            st.h_nrm = nrm.data();
            rc = fd2_boo_l2onehalf(p, na, go.data(), w.data(), prm->show_trigger, prm->change_weights_trigger,
                                   prm->max_iter, prm->prune_trigger, prm->n_prune, prm->n_beams_want, &st);
            result->trials += st.trials;
            result->phases += 1;
        }
        fd2_opt_problem_destroy(p);
        for (fd2_matrix* q : {ATs, As, Ds, DTs})
            if (q) fd2_matrix_destroy(q);
        if (rc) break;
        // DimReduction: rank by group norm, keep the strictly active beams
        std::vector<int64_t> rank(na);
        for (int64_t j = 0; j < na; j++) rank[j] = j;
        std::stable_sort(rank.begin(), rank.end(), [&](int64_t a, int64_t b) { return nrm[a] > nrm[b]; });
        const int64_t keep = std::min<int64_t>(na, std::max<int64_t>(0, (int64_t)st.num_active));
        std::vector<int64_t> next(keep);
        std::vector<float> w_next(keep), nrm_next(keep);
        int64_t off = 0;
        for (int64_t i = 0; i < keep && ce == cudaSuccess; i++) {
            const int64_t j = rank[i];
            next[i] = active[j];
            w_next[i] = w[j];
            nrm_next[i] = nrm[j];
            const int64_t len = go[j + 1] - go[j];
            if (len) {
                ce = cudaMemcpyAsync(xb[cur ^ 1] + off, xb[cur] + go[j], len * sizeof(float), cudaMemcpyDeviceToDevice,
                                     s);
                if (ce == cudaSuccess)
                    ce = cudaMemcpyAsync(vb[cur ^ 1] + off, vb[cur] + go[j], len * sizeof(float),
                                         cudaMemcpyDeviceToDevice, s);
            }
            off += len;
        }
        if (ce != cudaSuccess) {
            rc = FD2_ERR_CUDA;
            set_error("beam_orientation_optimization: %s", cudaGetErrorString(ce));
            break;
        }
        cur ^= 1;
        active = next;
        w = w_next;
        nrm = nrm_next;
        if (st.stop || keep == 0) {
            for (int64_t i = 0; i < keep; i++) {
                h_active[i] = (int32_t)active[i];
                h_norms[i] = nrm[i];
            }
            result->n_active = (int32_t)keep;
            result->iterations = st.k_global;
            ce = cudaMemcpyAsync(d_x, xb[cur], off * sizeof(float), cudaMemcpyDeviceToDevice, s);
            if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
            if (ce != cudaSuccess) {
                rc = FD2_ERR_CUDA;
                set_error("beam_orientation_optimization: %s", cudaGetErrorString(ce));
            }
            break;
        }
    }
    cudaStreamSynchronize(s);
    release();
    return rc;
}

}  // extern "C"
