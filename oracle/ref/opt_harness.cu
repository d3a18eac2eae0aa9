// opt_harness.cu -- extern "C" driver around the REFERENCE's own GPU optimizer
// (IMRTOpt/src/IMRTOptUtils.cu and IMRTOptimize_var1.cu, compiled whole, and
// the Eigen-free bodies IMRTOptimize.cu:16-194 (BOO_IMRT_L2OneHalf_gpu_QL) and
// :391-476 (polish_BOO_IMRT_gpu), compiled by line range), built by
// oracle/build_ref.sh into oracle/_ref/libfdref.so against the reference's
// unmodified headers and the Eigen stand-in under oracle/ref/eigen_stub.
// TEST INFRASTRUCTURE: pins the optimizer's oracle and the CUDA path (golden
// fixtures under tests/golden/).  Never linked by the product.
//
// Matrices arrive as host CSR (int64 offsets and columns, float values) and
// are uploaded the way IMRT::Eigen2Cusparse does (IMRTEigenLoad.cu:390-435):
// size_t offsets and columns, CUSPARSE_INDEX_64I, one SpMV buffer per matrix.
// Every entry point returns 0 on success; the reference's own error paths
// exit the process.
#include <cstdint>
#include <cstring>
#include <vector>

#include "IMRTOptimize.cuh"
#include "IMRTOptimize_var.cuh"

// One host CSR matrix as the callers pass it (the oracle's CSR layout).
struct RefCsr {
    int64_t rows, cols, nnz;
    const int64_t* offsets;
    const int64_t* columns;
    const float* values;
};

namespace {

// Upload of one CSR into a reference MatCSR64, as Eigen2Cusparse leaves it.
int upload(const RefCsr& s, IMRT::MatCSR64& d) {
    if (cudaMalloc((void**)&d.d_csr_offsets, (s.rows + 1) * sizeof(size_t)) != cudaSuccess) return 1;
    if (cudaMalloc((void**)&d.d_csr_columns, (s.nnz ? s.nnz : 1) * sizeof(size_t)) != cudaSuccess) return 1;
    if (cudaMalloc((void**)&d.d_csr_values, (s.nnz ? s.nnz : 1) * sizeof(float)) != cudaSuccess) return 1;
    cudaMemcpy(d.d_csr_offsets, s.offsets, (s.rows + 1) * sizeof(size_t), cudaMemcpyHostToDevice);
    if (s.nnz) {
        cudaMemcpy(d.d_csr_columns, s.columns, s.nnz * sizeof(size_t), cudaMemcpyHostToDevice);
        cudaMemcpy(d.d_csr_values, s.values, s.nnz * sizeof(float), cudaMemcpyHostToDevice);
    }
    checkCusparse(cusparseCreateCsr(&d.matA, s.rows, s.cols, s.nnz, d.d_csr_offsets, d.d_csr_columns,
                                    d.d_csr_values, CUSPARSE_INDEX_64I, CUSPARSE_INDEX_64I,
                                    CUSPARSE_INDEX_BASE_ZERO, CUDA_R_32F));
    d.numRows = s.rows;
    d.numCols = s.cols;
    d.nnz = s.nnz;
    IMRT::array_1d<float> in, out;
    IMRT::arrayInit(in, s.cols);
    IMRT::arrayInit(out, s.rows);
    cusparseHandle_t h;
    checkCusparse(cusparseCreate(&h));
    IMRT::bufferAllocate(d, in, out, h);
    checkCusparse(cusparseDestroy(h));
    return 0;
}

void to_device(IMRT::array_1d<float>& a, const float* src, size_t n) {
    IMRT::arrayInit(a, n);
    if (n) cudaMemcpy(a.data, src, n * sizeof(float), cudaMemcpyHostToDevice);
}

void to_host(float* dst, const IMRT::array_1d<float>& a) {
    if (a.size) cudaMemcpy(dst, a.data, a.size * sizeof(float), cudaMemcpyDeviceToHost);
}

// The fluence operator x2d of BeamOrientationOptimization (IMRTOptimize.cu:
// 325-337): one row per active beam, one column per fluence pixel, a 1 where
// the pixel's beamlet is on, in row-major order.
void x2d_host(int64_t n_beams, int64_t per_beam, const uint8_t* mask, std::vector<int64_t>& off,
              std::vector<int64_t>& col, std::vector<float>& val) {
    off.assign(1, 0);
    col.clear();
    val.clear();
    for (int64_t b = 0; b < n_beams; b++) {
        for (int64_t j = 0; j < per_beam; j++)
            if (mask[b * per_beam + j] > 0) {
                col.push_back(j);
                val.push_back(1.0f);
            }
        off.push_back((int64_t)col.size());
    }
}

struct Problem {
    IMRT::MatCSR64 A, AT, D, DT;
    IMRT::array_1d<float> maxDose, minDoseTarget, minDoseTargetWeights, maxWeightsLong, OARWeightsLong;
    size_t n_ptv = 0, n_oar = 0;
    float gamma = 1.0f, eta = 0.1f;
};

}  // namespace

extern "C" {

void* ref_opt_problem_create(const RefCsr* A, const RefCsr* AT, const RefCsr* D, const RefCsr* DT, int64_t n_ptv,
                             int64_t n_oar, const float* max_dose, const float* max_weights, const float* min_dose,
                             const float* min_weights, const float* oar_weights, float gamma, float eta) {
    Problem* p = new Problem;
    if (upload(*A, p->A) || upload(*AT, p->AT) || upload(*D, p->D) || upload(*DT, p->DT)) {
        delete p;
        return nullptr;
    }
    p->n_ptv = n_ptv;
    p->n_oar = n_oar;
    p->gamma = gamma;
    p->eta = eta;
    to_device(p->maxDose, max_dose, n_ptv + n_oar);
    to_device(p->maxWeightsLong, max_weights, n_ptv + n_oar);
    to_device(p->minDoseTarget, min_dose, n_ptv);
    to_device(p->minDoseTargetWeights, min_weights, n_ptv);
    to_device(p->OARWeightsLong, oar_weights, n_oar);
    return p;
}

void ref_opt_problem_destroy(void* h) { delete (Problem*)h; }

// eval_g::evaluate (IMRTOptUtils.cu:74-156)
int ref_opt_eval_g(void* h, const float* x, float* out) {
    Problem& p = *(Problem*)h;
    cusparseHandle_t hs;
    cublasHandle_t hb;
    checkCusparse(cusparseCreate(&hs));
    checkCublas(cublasCreate(&hb));
    {
        IMRT::eval_g op(p.n_ptv, p.n_oar, p.D.numRows);
        IMRT::array_1d<float> xd;
        to_device(xd, x, p.A.numCols);
        *out = op.evaluate(p.A, p.D, xd, p.gamma, hs, hb, p.maxDose.data, p.minDoseTarget.data,
                           p.minDoseTargetWeights.data, p.maxWeightsLong.data, p.OARWeightsLong.data, p.eta);
    }
    cublasDestroy(hb);
    cusparseDestroy(hs);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
}

// eval_grad::evaluate (IMRTOptUtils.cu:512-631)
int ref_opt_eval_grad(void* h, const float* x, float* out, float* grad) {
    Problem& p = *(Problem*)h;
    cusparseHandle_t hs;
    cublasHandle_t hb;
    checkCusparse(cusparseCreate(&hs));
    checkCublas(cublasCreate(&hb));
    {
        IMRT::eval_grad op(p.n_ptv, p.n_oar, p.D.numRows, p.A.numCols);
        IMRT::array_1d<float> xd, g;
        to_device(xd, x, p.A.numCols);
        IMRT::arrayInit(g, p.A.numCols);
        *out = op.evaluate(p.A, p.AT, p.D, p.DT, xd, g, p.gamma, hs, hb, p.maxDose.data, p.minDoseTarget.data,
                           p.minDoseTargetWeights.data, p.maxWeightsLong.data, p.OARWeightsLong.data, p.eta);
        to_host(grad, g);
    }
    cublasDestroy(hb);
    cusparseDestroy(hs);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
}

// proxL2Onehalf_QL_gpu::customInit/evaluate (IMRTOptimize_var1.cu:457-541) on
// the beam x pixel operator of `mask` holding g0's values in row-major order.
int ref_opt_prox(int64_t n_beams, int64_t per_beam, const uint8_t* mask, const float* g0, const float* tau,
                 float* prox, float* nrm) {
    std::vector<int64_t> off, col;
    std::vector<float> val;
    x2d_host(n_beams, per_beam, mask, off, col, val);
    const int64_t nnz = (int64_t)col.size();
    std::memcpy(val.data(), g0, nnz * sizeof(float));
    RefCsr s{n_beams, per_beam, nnz, off.data(), col.data(), val.data()};
    cusparseHandle_t hs;
    checkCusparse(cusparseCreate(&hs));
    {
        IMRT::MatCSR64 g, out;
        if (upload(s, g) || upload(s, out)) return 1;
        IMRT::array_1d<float> t, n;
        to_device(t, tau, n_beams);
        IMRT::arrayInit(n, n_beams);
        IMRT::proxL2Onehalf_QL_gpu op;
        op.customInit(g, hs);
        op.evaluate(g, t, out, n, hs);
        cudaMemcpy(prox, out.d_csr_values, nnz * sizeof(float), cudaMemcpyDeviceToHost);
        to_host(nrm, n);
    }
    cusparseDestroy(hs);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
}

// Both forms of beamWeightsInit_func: the host one BeamOrientationOptimization
// calls (IMRTOptimize_var1.cu:125-161, Eigen sparse x dense) into out_host,
// and the cuSPARSE/cuBLAS one (:49-122) into out_gpu.  blocks[b] is beam b's
// VOI x beamlets matrix.
int ref_opt_beam_weights(int64_t n_beams, const RefCsr* blocks, int64_t n_ptv, int64_t n_oar, float* out_host,
                         float* out_gpu) {
    std::vector<IMRT::MatCSR_Eigen> mats(n_beams);
    std::vector<const IMRT::MatCSR_Eigen*> ptrs(n_beams);
    std::vector<std::vector<int64_t>> offs(n_beams), cols(n_beams);
    std::vector<std::vector<float>> vals(n_beams);
    for (int64_t b = 0; b < n_beams; b++) {
        const RefCsr& s = blocks[b];
        offs[b].assign(s.offsets, s.offsets + s.rows + 1);
        cols[b].assign(s.columns, s.columns + s.nnz);
        vals[b].assign(s.values, s.values + s.nnz);
        mats[b].harness_view(s.rows, s.cols, offs[b].data(), cols[b].data(), vals[b].data(), s.nnz);
        ptrs[b] = &mats[b];
    }
    Eigen::VectorXf w;
    if (IMRT::beamWeightsInit_func(ptrs, w, n_ptv, n_oar)) return 1;
    for (int64_t b = 0; b < n_beams; b++) out_host[b] = w(b);

    cusparseHandle_t hs;
    cublasHandle_t hb;
    checkCusparse(cusparseCreate(&hs));
    checkCublas(cublasCreate(&hb));
    int rc = 0;
    {
        IMRT::MatReservior res;
        res.reservior.resize(n_beams);
        for (int64_t b = 0; b < n_beams && !rc; b++) rc = upload(blocks[b], res.reservior[b]);
        IMRT::array_1d<float> wd;
        IMRT::arrayInit(wd, n_beams);
        if (!rc) rc = IMRT::beamWeightsInit_func(res, wd, n_ptv, n_oar, hs, hb) ? 1 : 0;
        if (!rc) to_host(out_gpu, wd);
    }
    cublasDestroy(hb);
    cusparseDestroy(hs);
    if (rc) return rc;
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
}

// BOO_IMRT_L2OneHalf_gpu_QL (IMRTOptimize.cu:16-194): one prune phase.
// In/out: beam_weights[n_beams], xkm1/vkm1[n], *k_global, *theta_km1, *tkm1.
// loss[iters_global] is in/out: the iterations run fill their entries.
// Out: nrm[n_beams], *num_active,
// *stop.  mask is the [n_beams][per_beam] fluence map of the phase's beams.
int ref_opt_boo(void* h, int64_t n_beams, int64_t per_beam, const uint8_t* mask, float* beam_weights,
                int show_trigger, int change_trigger, int iters_global, const int* prune, int n_prune, int want,
                int* k_global, float* theta_km1, float* tkm1, float* xkm1, float* vkm1, float* loss, float* nrm,
                float* num_active, int* stop) {
    Problem& p = *(Problem*)h;
    const size_t n = p.A.numCols;
    std::vector<int64_t> off, col;
    std::vector<float> val;
    x2d_host(n_beams, per_beam, mask, off, col, val);
    if ((size_t)col.size() != n) return 3;
    RefCsr xs{n_beams, per_beam, (int64_t)col.size(), off.data(), col.data(), val.data()};
    int rc = 0;
    {
        IMRT::MatCSR64 x2d, x2dprox;
        if (upload(xs, x2d) || upload(xs, x2dprox)) return 1;
        IMRT::array_1d<float> w, x, v;
        to_device(w, beam_weights, n_beams);
        to_device(x, xkm1, n);
        to_device(v, vkm1, n);
        std::vector<int> pr(prune, prune + n_prune);
        std::vector<float> loss_v(loss, loss + iters_global), nrm_v(n_beams, 0.0f);
        float active = 0.0f;
        bool st = false;
        rc = IMRT::BOO_IMRT_L2OneHalf_gpu_QL(p.A, p.AT, p.D, p.DT, w, p.maxDose, p.minDoseTarget,
                                             p.minDoseTargetWeights, p.maxWeightsLong, p.OARWeightsLong, per_beam,
                                             p.gamma, p.eta, show_trigger, change_trigger, *k_global, iters_global,
                                             pr, want, *theta_km1, *tkm1, x, v, x2d, x2dprox, loss_v, nrm_v,
                                             active, st)
                 ? 1
                 : 0;
        to_host(beam_weights, w);
        to_host(xkm1, x);
        to_host(vkm1, v);
        std::memcpy(loss, loss_v.data(), iters_global * sizeof(float));
        std::memcpy(nrm, nrm_v.data(), n_beams * sizeof(float));
        *num_active = active;
        *stop = st ? 1 : 0;
    }
    if (rc) return rc;
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
}

// polish_BOO_IMRT_gpu (IMRTOptimize.cu:391-476).
int ref_opt_polish(void* h, int iters_global, int iters_local, int* k_global, float* theta_km1, float* tkm1,
                   float* xkm1, float* vkm1, float* loss) {
    Problem& p = *(Problem*)h;
    const size_t n = p.A.numCols;
    int rc = 0;
    {
        IMRT::array_1d<float> x, v;
        to_device(x, xkm1, n);
        to_device(v, vkm1, n);
        std::vector<float> loss_v(loss, loss + iters_global);
        rc = IMRT::polish_BOO_IMRT_gpu(p.A, p.AT, p.D, p.DT, p.maxDose, p.minDoseTarget, p.minDoseTargetWeights,
                                       p.maxWeightsLong, p.OARWeightsLong, p.gamma, p.eta, *k_global, iters_global,
                                       iters_local, *theta_km1, *tkm1, x, v, loss_v)
                 ? 1
                 : 0;
        to_host(xkm1, x);
        to_host(vkm1, v);
        std::memcpy(loss, loss_v.data(), iters_global * sizeof(float));
    }
    if (rc) return rc;
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
}

// DimReduction (IMRTOptUtils.cu:726-793) after a phase: active[n_active] (in:
// the phase's beams, out: the kept ones, strongest first), beam_cols[n_all]
// the beamlet count of every beam.  Out: weights_out, x_out, v_out of the
// kept beams, *n_kept.
int ref_opt_dim_reduction(int n_active, int* active, int n_all, const int64_t* beam_cols, const float* weights,
                          const float* xkm1, const float* vkm1, int64_t n, const float* nrm, int n_keep,
                          float* weights_out, float* x_out, float* v_out, int* n_kept) {
    std::vector<IMRT::MatCSR_Eigen> voi(n_all);
    for (int b = 0; b < n_all; b++) voi[b].harness_view(0, beam_cols[b], nullptr, nullptr, nullptr, 0);
    std::vector<int> act(active, active + n_active);
    Eigen::VectorXf w_cpu, x_cpu, v_cpu;
    int rc = 0;
    {
        IMRT::array_1d<float> w, x, v;
        to_device(w, weights, n_active);
        to_device(x, xkm1, n);
        to_device(v, vkm1, n);
        std::vector<float> nrm_v(nrm, nrm + n_active);
        rc = IMRT::DimReduction(act, w_cpu, x_cpu, v_cpu, w, x, v, nrm_v, n_keep, voi) ? 1 : 0;
    }
    if (rc) return rc;
    *n_kept = (int)act.size();
    for (size_t i = 0; i < act.size(); i++) {
        active[i] = act[i];
        weights_out[i] = w_cpu(i);
    }
    std::memcpy(x_out, x_cpu.data(), x_cpu.size() * sizeof(float));
    std::memcpy(v_out, v_cpu.data(), v_cpu.size() * sizeof(float));
    return 0;
}

// The C library's rand() stream the reference seeds (std::srand(10086),
// IMRTOptimize.cu:240-243; arrayRand01, IMRTOptUtils.cu:246-253), for fixtures.
void ref_opt_rand01(unsigned seed, int reseed, int64_t n, float* out) {
    if (reseed) std::srand(seed);
    for (int64_t i = 0; i < n; i++) out[i] = (float)std::rand() / RAND_MAX;
}

}  // extern "C"
