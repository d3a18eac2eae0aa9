"""The reference's C++ names (include/fd2_compat.hpp) driven from C++ on the
GPU: a caller built with g++ runs fastdose::TermaComputeCollective,
fastdose::DoseComputeCollective (FastDoseLib/include/TermaComp.cuh:7-17,
DoseComp.cuh:9-19) on its own cudaMalloc'd BEV buffers and
IMRT::DoseMatConstruction (IMRTOpt/include/IMRTDoseMat.cuh:71-78), and its
results equal the same calls made through the C ABI from Python, bit for bit."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from fastdose_b200 import _lib, api
from fastdose_b200.types import BEAM_DTYPE, VOLUME_DTYPE
from plan_cases import small_case

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CALLER = r"""
#include "fd2_compat.hpp"
#include <cstdio>
#include <vector>

template <class T> static std::vector<T> load(const char* dir, const char* name) {
    char p[4096];
    std::snprintf(p, sizeof p, "%s/%s", dir, name);
    FILE* f = std::fopen(p, "rb");
    std::fseek(f, 0, SEEK_END);
    long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    std::vector<T> v(n / sizeof(T));
    if (std::fread(v.data(), sizeof(T), v.size(), f) != v.size()) v.clear();
    std::fclose(f);
    return v;
}
template <class T> static void save(const char* dir, const char* name, const T* p, size_t n) {
    char q[4096];
    std::snprintf(q, sizeof q, "%s/%s", dir, name);
    FILE* f = std::fopen(q, "wb");
    std::fwrite(p, sizeof(T), n, f);
    std::fclose(f);
}
#define CHECK(x) do { if (x) { std::printf("failed: %s: %s\n", #x, fd2_last_error()); return 1; } } while (0)

int main(int argc, char** argv) {
    const char* dir = argv[1];
    auto beams = load<fd2_beam_t>(dir, "beams.bin");
    auto dens = load<float>(dir, "density.bin");
    auto volv = load<fd2_volume_t>(dir, "volume.bin");
    auto spec = load<float>(dir, "spectrum.bin");   // E, fluence, mu, mu_en (n each)
    auto kern = load<float>(dir, "kernel.bin");     // theta, A, a, B, b (nt each), then phi (np)
    auto flu = load<float>(dir, "fluence.bin");
    auto dims = load<int>(dir, "dims.bin");         // n_spec, n_theta, n_phi
    const int ns = dims[0], nt = dims[1], np_ = dims[2];
    fd2_context* ctx = nullptr;
    CHECK(fd2_context_create(0, &ctx));
    fd2_density* d = nullptr;
    fd2_spectrum* sp = nullptr;
    fd2_cccs_kernel* k = nullptr;
    CHECK(fd2_density_create(ctx, dens.data(), &volv[0], &d));
    CHECK(fd2_spectrum_create(ctx, ns, &spec[0], &spec[ns], &spec[2 * ns], &spec[3 * ns], &sp));
    CHECK(fd2_kernel_create(ctx, nt, &kern[0], &kern[nt], &kern[2 * nt], &kern[3 * nt], &kern[4 * nt], np_,
                            &kern[5 * nt], &k));
    const size_t n = beams.size(), P = (size_t)beams[0].fmap_size[0] * beams[0].fmap_size[1];
    std::vector<size_t> off(n + 1, 0);
    for (size_t i = 0; i < n; i++) off[i + 1] = off[i] + (size_t)beams[i].long_dim * P;
    float *T, *R, *D, *F;
    fd2_beam_t* db;
    cudaMalloc(&T, off[n] * 4); cudaMalloc(&R, off[n] * 4); cudaMalloc(&D, off[n] * 4); cudaMalloc(&F, P * 4);
    cudaMemset(D, 0, off[n] * 4);
    cudaMalloc(&db, n * sizeof(fd2_beam_t));
    cudaMemcpy(db, beams.data(), n * sizeof(fd2_beam_t), cudaMemcpyHostToDevice);
    cudaMemcpy(F, flu.data(), P * 4, cudaMemcpyHostToDevice);
    std::vector<float*> hT(n), hR(n), hD(n), hF(n, F);
    for (size_t i = 0; i < n; i++) { hT[i] = T + off[i]; hR[i] = R + off[i]; hD[i] = D + off[i]; }
    float **aT, **aR, **aD, **aF;
    cudaMalloc(&aT, n * 8); cudaMalloc(&aR, n * 8); cudaMalloc(&aD, n * 8); cudaMalloc(&aF, n * 8);
    cudaMemcpy(aT, hT.data(), n * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(aR, hR.data(), n * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(aD, hD.data(), n * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(aF, hF.data(), n * 8, cudaMemcpyHostToDevice);
    CHECK(fastdose::TermaComputeCollective(P, n, db, aF, aT, aR, ctx, d, sp, 0));
    CHECK(fastdose::DoseComputeCollective(P, n, db, aT, aR, aD, ctx, k, 0));
    CHECK(cudaDeviceSynchronize() != cudaSuccess);
    std::vector<float> hd(off[n]);
    cudaMemcpy(hd.data(), D, off[n] * 4, cudaMemcpyDeviceToHost);
    save(dir, "dose_bev.bin", hd.data(), hd.size());

    fd2_dosemat_params_t prm;
    fd2_dosemat_params_default(&prm);
    fd2_csr_ensemble* ens = nullptr;
    CHECK(IMRT::DoseMatConstruction(ctx, {(uint32_t)n}, beams, flu, d, sp, k, prm, &ens, 0));
    fd2_csr_info_t info;
    CHECK(fd2_csr_ensemble_info(ens, &info));
    std::vector<int64_t> ro(info.n_rows + 1);
    std::vector<int32_t> col(info.nnz);
    std::vector<float> val(info.nnz);
    CHECK(fd2_csr_ensemble_to_host(ens, ro.data(), col.data(), val.data()));
    save(dir, "row_off.bin", ro.data(), ro.size());
    save(dir, "col.bin", col.data(), col.size());
    save(dir, "val.bin", val.data(), val.size());
    fd2_csr_ensemble_destroy(ens);
    fd2_kernel_destroy(k); fd2_spectrum_destroy(sp); fd2_density_destroy(d);
    cudaFree(T); cudaFree(R); cudaFree(D); cudaFree(F); cudaFree(db);
    cudaFree(aT); cudaFree(aR); cudaFree(aD); cudaFree(aF);
    fd2_context_destroy(ctx);
    std::printf("ok %zu beamlets, nnz %llu\n", n, (unsigned long long)info.nnz);
    return 0;
}
"""


def test_cpp_caller_matches_the_c_abi(ctx, tmp_path):
    if not shutil.which("g++"):
        pytest.skip("no g++")
    case = small_case()
    ph, spec, kern = case["phantom"], case["spectrum"], case["kernel"]
    beams = np.ascontiguousarray(case["beams"], BEAM_DTYPE).copy()
    P = int(beams[0]["fmap_size"][0]) * int(beams[0]["fmap_size"][1])
    beams["TermaBEV_pitch"] = beams["DensityBEV_pitch"] = P * 4
    d = tmp_path
    beams.tofile(d / "beams.bin")
    np.ascontiguousarray(ph.density, np.float32).tofile(d / "density.bin")
    np.asarray(ph.volume, VOLUME_DTYPE).reshape(1).tofile(d / "volume.bin")
    np.concatenate([spec.energy, spec.fluence, spec.mu, spec.mu_en]).astype(np.float32).tofile(d / "spectrum.bin")
    np.concatenate([kern.theta, kern.A, kern.a, kern.B, kern.b, kern.phi]).astype(np.float32).tofile(d / "kernel.bin")
    np.asarray(case["fluence"], np.float32).tofile(d / "fluence.bin")
    np.array([spec.n, kern.n_theta, kern.n_phi], np.int32).tofile(d / "dims.bin")
    src = d / "caller.cpp"
    src.write_text(CALLER)
    exe = d / "caller"
    libdir = os.path.dirname(_lib.LIB_PATH)
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include",
                    str(src), "-L", libdir, "-lfd2", "-L", "/usr/local/cuda/lib64", "-lcudart",
                    f"-Wl,-rpath,{libdir}", "-Wl,-rpath,/usr/local/cuda/lib64", "-o", str(exe)], check=True)
    out = subprocess.run([str(exe), str(d)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0 and out.stdout.startswith("ok"), out.stdout + out.stderr

    # the same calls through the C ABI from Python
    import torch

    dens, sp, kn = api.Density(ctx, ph.density, ph.volume), api.Spectrum(ctx, spec), api.Kernel(ctx, kern)
    batch = api.BEVBatch(beams)
    api.TermaComputeCollective(ctx, batch, case["fluence"], dens, sp)
    api.DoseComputeCollective(ctx, batch, kn)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(np.fromfile(d / "dose_bev.bin", np.float32), batch.dose.cpu().numpy())
    m = api.DoseMatConstruction(ctx, [beams], case["fluence"], dens, sp, kn)
    ro, col, val = m.to_host()
    np.testing.assert_array_equal(np.fromfile(d / "row_off.bin", np.int64), ro)
    np.testing.assert_array_equal(np.fromfile(d / "col.bin", np.int32), col)
    np.testing.assert_array_equal(np.fromfile(d / "val.bin", np.float32), val)
