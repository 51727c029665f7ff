"""The C++ drop-in header compiles in a host program written the way the
reference's driver uses src/ntt_config.h, links against libntt_b200.so, and
reports the reference's default configuration (no GPU needed).  A second
client, marked gpu, runs launch_ntt<DefaultNTTLaunchConfig<16>> and
launch_intt<...> on the reference's Montgomery-form tables exactly as the
reference's driver does (src/v04_montgomery.cu:985 and :1034) and is checked
word for word against the oracle."""
import os
import shutil
import subprocess

import pytest

from oracle import oracle as O

ROOT = os.path.join(os.path.dirname(__file__), "..")

CLIENT = r"""
#include <cstdio>
#include "ntt_b200_config.hpp"

template <typename LC> void print_transform() {
    TransformConfig t = LC::runtime_transform();
    std::printf("%d %d %d %d %d %d %d %d %d %d %d %d %d\n", LC::logN,
        t.ntt_phase1.radix_stages, t.ntt_phase1.stage_merging, t.ntt_phase1.warp_batching,
        t.ntt_phase2.radix_stages, t.ntt_phase2.stage_merging, t.ntt_phase2.warp_batching,
        t.intt_phase1.radix_stages, t.intt_phase1.stage_merging, t.intt_phase1.warp_batching,
        t.intt_phase2.radix_stages, t.intt_phase2.stage_merging, t.intt_phase2.warp_batching);
}

int main() {
    VersionConfig v = default_ntt_config();
    std::printf("%d %zu\n", v.logN, v.moduli.size());
    for (const ModulusConfig& m : v.moduli) std::printf("%u %u\n", m.qi, m.primitive_root);
    print_transform<DefaultNTTLaunchConfig<12>>();
    print_transform<DefaultNTTLaunchConfig<16>>();
    print_transform<DefaultNTTLaunchConfig<17>>();
    // launchers must instantiate with the reference's argument list
    auto* f = &launch_ntt<DefaultNTTLaunchConfig<16>>;
    auto* g = &launch_intt<DefaultNTTLaunchConfig<16>>;
    std::printf("%d\n", f != nullptr && g != nullptr);
    return 0;
}
"""


@pytest.fixture(scope="module")
def client(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    d = tmp_path_factory.mktemp("cfg")
    src = d / "client.cpp"
    src.write_text(CLIENT)
    exe = d / "client"
    libdir = os.path.abspath(os.path.join(ROOT, "ntt_b200"))
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), str(src),
                    "-L", libdir, "-lntt_b200", "-Wl,-rpath," + libdir, "-o", str(exe)],
                   check=True)
    return subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")


def test_default_version_config(client):
    logN, count = map(int, client[0].split())
    assert (logN, count) == (16, 16)
    mods = [tuple(map(int, l.split())) for l in client[1:1 + count]]
    assert mods == O.REFERENCE_DEFAULT_MODULI


def test_default_launch_configs(client):
    rows = [list(map(int, l.split())) for l in client[17:20]]
    assert rows[0] == [12, 3, 3, 4, 9, 3, 0, 9, 3, 0, 3, 3, 4]
    assert rows[1] == [16, 7, 4, 4, 9, 3, 0, 9, 3, 0, 7, 4, 4]
    assert rows[2] == [17, 8, 3, 4, 9, 3, 0, 9, 3, 0, 8, 3, 4]
    assert client[20] == "1"


GPU_CLIENT = r"""
#include <cstdio>
#include <cstdlib>
#include <vector>
#include <cuda_runtime.h>
#include "ntt_b200_config.hpp"

// in: N*L input words, tw, itw (N*L each), q, q_inv, r2, degree_inv (L each)
// out: forward result, then the inverse of it (2*N*L words)
int main(int argc, char** argv) {
    using LC = DefaultNTTLaunchConfig<16>;
    const size_t N = size_t{1} << LC::logN, L = 16, W = N * L;
    std::vector<uint32_t> in(3 * W + 4 * L), out(2 * W);
    FILE* f = std::fopen(argv[1], "rb");
    if (!f || std::fread(in.data(), 4, in.size(), f) != in.size()) return 2;
    std::fclose(f);
    uint32_t *A, *tw, *itw, *q, *qi, *r2, *di;
    cudaMalloc(&A, W * 4); cudaMalloc(&tw, W * 4); cudaMalloc(&itw, W * 4);
    cudaMalloc(&q, L * 4); cudaMalloc(&qi, L * 4); cudaMalloc(&r2, L * 4); cudaMalloc(&di, L * 4);
    cudaMemcpy(A, in.data(), W * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(tw, in.data() + W, W * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(itw, in.data() + 2 * W, W * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(q, in.data() + 3 * W, L * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(qi, in.data() + 3 * W + L, L * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(r2, in.data() + 3 * W + 2 * L, L * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(di, in.data() + 3 * W + 3 * L, L * 4, cudaMemcpyHostToDevice);
    if (launch_ntt<LC>(A, tw, q, qi, r2, L) != NTT_OK) return 3;
    if (cudaDeviceSynchronize() != cudaSuccess) return 4;
    cudaMemcpy(out.data(), A, W * 4, cudaMemcpyDeviceToHost);
    if (launch_intt<LC>(A, itw, q, qi, di, L) != NTT_OK) return 5;
    if (cudaDeviceSynchronize() != cudaSuccess) return 6;
    cudaMemcpy(out.data() + W, A, W * 4, cudaMemcpyDeviceToHost);
    f = std::fopen(argv[2], "wb");
    if (!f || std::fwrite(out.data(), 4, out.size(), f) != out.size()) return 7;
    std::fclose(f);
    return 0;
}
"""


@pytest.mark.gpu
def test_cpp_dropin_launchers_on_gpu(tmp_path, torch_cuda):
    """launch_ntt / launch_intt templates of the C++ drop-in header, called
    from C++ with the reference's tables and default moduli, give the
    oracle's forward words and then the input back."""
    import numpy as np
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    src = tmp_path / "gpu_client.cpp"
    src.write_text(GPU_CLIENT)
    exe = tmp_path / "gpu_client"
    libdir = os.path.abspath(os.path.join(ROOT, "ntt_b200"))
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
                    "-I", os.path.join(cuda, "include"), str(src), "-L", libdir, "-lntt_b200",
                    "-L", os.path.join(cuda, "lib64"), "-lcudart", "-Wl,-rpath," + libdir,
                    "-o", str(exe)], check=True)
    mods = O.REFERENCE_DEFAULT_MODULI
    T = O.LimbTables(16, mods)
    tw, itw = T.mont_tables()
    x = O.fill_random_ref_compatible(16, T.q)
    blob = np.concatenate([a.astype(np.uint32).reshape(-1) for a in
                           (x, tw, itw, T.q, T.q_inv, T.r2, T.degree_inv_mont)])
    (tmp_path / "in.bin").write_bytes(blob.tobytes())
    r = subprocess.run([str(exe), str(tmp_path / "in.bin"), str(tmp_path / "out.bin")],
                       capture_output=True, text=True)
    assert r.returncode == 0, (r.returncode, r.stderr)
    out = np.frombuffer((tmp_path / "out.bin").read_bytes(), dtype=np.uint32)
    W = x.size
    assert np.array_equal(out[:W], T.forward_mont(x, os.cpu_count() or 4).reshape(-1))
    assert np.array_equal(out[W:], x.reshape(-1))
