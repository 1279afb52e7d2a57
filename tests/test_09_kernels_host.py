"""The FFT passes of the MD step, the kernels themselves, emulated on the host.

`tests/host_emu/xy_emu.cpp` compiles `feram_b200/csrc/fg_kernels.cuh` with
g++ behind `tests/host_emu/kernel_emu.h` (the threads of a block as fibers
switched at __syncthreads() and warp shuffles, blocks in grid order) and runs
the library's own kernels on small supercells:

* `k_xy_fwd` (SRC_U9: u and u⊗u formed on load, dipoFFT.F:19-44; with the
  acoustic displacement as components 9..11, or Z*(R) u for per-site Z*,
  dipoFFT.F:36-44) against a direct 2D DFT per z plane and component, in the
  slot orders of the x and y plans; `k_xy_inv` must return Lx*Ly times each
  plane;
* the 3-component r2c / c2r of `fg_fft_r2c3` / `fg_fft_c2r3` (`k_xy_fwd`
  SRC_FIELD + `k_z_pass`, coord_module.F:155-157,310-312) against a direct 3D
  DFT, and back to Lx*Ly*Lz times the fields;

for every compile-time instance of the library's dispatch (the xy passes of
16³ to 128³, 24³ and 48³ planes, the z passes of Lz = 16 to 128, 24, 48) and
for runtime plans with radices 3 and 5 and odd Lx/2, in FP64 and FP32.  No
GPU; the same kernels run on the B200 in test_50 and test_70."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "host_emu", "xy_emu.cpp")
CUDA_INC = "/usr/local/cuda/include"

# relative errors; any index or twiddle mistake gives errors of order one
TOL = {"f64": 4e-15, "f32": 2e-6}


@pytest.fixture(scope="module")
def emu_lines(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None or not os.path.isdir(CUDA_INC):
        pytest.skip("needs g++ and the CUDA headers")
    exe = str(tmp_path_factory.mktemp("kernemu") / "xy_emu")
    subprocess.run([gxx, "-std=c++20", "-O1", "-I", CUDA_INC, "-I", os.path.join(ROOT, "feram_b200", "csrc"),
                    "-I", os.path.join(ROOT, "include"), "-I", os.path.dirname(SRC), SRC, "-o", exe],
                   check=True, capture_output=True, text=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True, timeout=600).stdout
    rows = {}
    for line in out.splitlines():
        name, ef, eb = line.split()
        rows[name] = (float(ef), float(eb))
    return rows


def test_every_instance_ran(emu_lines):
    for prec in ("f64", "f32"):
        for L in (16, 24, 32, 48, 64, 128):
            assert f"xy_{prec}_ct_{L}x{L}x" in " ".join(emu_lines)
        for name in ("fft3_{p}_ct_16x16x16", "fft3_{p}_ct_16x16x128", "fft3_{p}_ct_24x24x24", "fft3_{p}_ct_16x16x48",
                     "fft3_{p}_rt_20x6x15", "xy_{p}_rt_10x6x2"):
            assert name.format(p=prec) in emu_lines
        for name in ("xy_{p}_ct_16x16x2_acou", "xy_{p}_ct_16x16x2_zstar", "xy_{p}_rt_12x10x2_zstar"):
            assert name.format(p=prec) in emu_lines
    assert len(emu_lines) == 2 * (15 + 8)


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_forward_passes_give_the_dft(emu_lines, prec):
    bad = {n: v for n, v in emu_lines.items() if f"_{prec}_" in n and not v[0] <= TOL[prec]}
    assert not bad, bad


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_inverse_passes_return_the_fields(emu_lines, prec):
    bad = {n: v for n, v in emu_lines.items() if f"_{prec}_" in n and not v[1] <= TOL[prec]}
    assert not bad, bad
