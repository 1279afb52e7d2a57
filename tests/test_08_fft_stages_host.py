"""The shared-memory FFT stages of the device code, emulated on the host.

`feram_b200/csrc/fft_smem.cuh` is compiled with g++ (`tests/host_emu/
fft_stages_emu.cpp`, CUDA built-ins replaced by `emu_shim.h`) and every
thread of a stage is run in turn, stage after stage: the device's own index
arithmetic, stage plans and radix kernels, checked against an exact DFT with
no GPU.  Covered: the compile-time lengths of the xy and z kernels (4 to 512,
12, 24, 48; rows, interleaved columns and the z tile's padded component
layout), the stages fused with global loads and stores (`ct_stage_io`), and
runtime plans of radices 2-5, 8 and 16 in both orders.  The forward result
is read in digit-reversed order (decimation in frequency: the frequencies
k = s mod r of a radix-r stage land in its s-th sub-block), which is the
order the k-space tables and the z kernel assume; the inverse must return
n times the input.  The device FFT itself is checked on the GPU against
numpy and cuFFT (test_50, test_52)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "host_emu", "fft_stages_emu.cpp")
CUDA_INC = "/usr/local/cuda/include"

# relative errors: FP64 a few ulps of the largest term, FP32 likewise
TOL = {"f64": 2e-15, "f32": 1e-6}


@pytest.fixture(scope="module")
def emu_lines(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None or not os.path.isdir(CUDA_INC):
        pytest.skip("needs g++ and the CUDA headers")
    exe = str(tmp_path_factory.mktemp("fftemu") / "fft_stages_emu")
    subprocess.run([gxx, "-std=c++17", "-O1", "-I", CUDA_INC, "-I", os.path.join(ROOT, "feram_b200", "csrc"),
                    "-I", os.path.dirname(SRC), SRC, "-o", exe], check=True, capture_output=True, text=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    rows = {}
    for line in out.splitlines():
        name, ef, eb = line.split()
        rows[name] = (float(ef), float(eb))
    return rows


def test_every_case_ran(emu_lines):
    kinds = {n.split("_")[0] for n in emu_lines}
    assert kinds == {"ct", "io", "rt"}
    # 18 compile-time layouts, 4 fused-io cases, 80 runtime plans per precision
    assert len(emu_lines) == 2 * (18 + 4 + 80)
    for n in (4, 8, 16, 32, 64, 128, 256, 512, 12, 24, 48):
        assert f"ct_f32_rows_n{n}" in emu_lines and f"ct_f64_rows_n{n}" in emu_lines


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_stages_give_the_dft_in_digit_reversed_order(emu_lines, prec):
    bad = {n: v for n, v in emu_lines.items() if f"_{prec}_" in n and v[0] > TOL[prec]}
    assert not bad, bad


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_inverse_stages_return_n_times_the_input(emu_lines, prec):
    bad = {n: v for n, v in emu_lines.items() if f"_{prec}_" in n and v[1] > TOL[prec]}
    assert not bad, bad
