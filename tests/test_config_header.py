"""The C++ drop-in header compiles in a host program written the way the
reference's driver uses src/ntt_config.h, links against libntt_b200.so, and
reports the reference's default configuration.  Runs without a GPU."""
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
