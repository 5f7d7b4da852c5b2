"""The drop-in C++ API (include/lifted.hpp, the four lifted::lwt overloads of
the reference's src/lifted.hpp:13-39) run on the GPU: a small C++ program
compiled against the header and liblifted_b200.so calls every overload on
host vectors and on cudaMalloc'd device pointers, as the reference's own
driver tests call lwt (tests/test_dwt.cpp:158,222), and writes the outputs to
files that are compared here with the oracle, bit for bit."""
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

import pyoracle as po

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from lifted_b200 import _lib  # noqa: E402

ROOT = Path(__file__).resolve().parents[1]
CUDA = Path("/usr/local/cuda")

PROGRAM = r"""
#include <cuda_runtime.h>

#include <cstdio>
#include <string>
#include <vector>

#include "lifted.hpp"

using namespace lifted;

template <typename T>
std::vector<T> load(const std::string& path, size_t n) {
  std::vector<T> v(n);
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f || std::fread(v.data(), sizeof(T), n, f) != n) std::exit(10);
  std::fclose(f);
  return v;
}

template <typename T>
void save(const std::string& path, const std::vector<T>& v) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f || std::fwrite(v.data(), sizeof(T), v.size(), f) != v.size()) std::exit(11);
  std::fclose(f);
}

// Forward then ForwardAdjoint of a separable 2D transform, on host vectors
// and on device pointers.
template <typename T>
void separable(const std::string& dir, const char* tag) {
  const size_t n = 512;
  const size_v shape{n, n}, axes{0, 1}, levels{6, 6};
  const stride_v st{(ptrdiff_t)n, 1};
  std::vector<T> x = load<T>(dir + "/x_" + tag + ".bin", n * n), y(n * n), z(n * n);
  lwt(Wavelet::CDF9_7, Transform::Forward, BoundaryCondition::Zero, shape, st, st, axes,
      levels, x.data(), y.data());
  lwt(Wavelet::CDF9_7, Transform::ForwardAdjoint, BoundaryCondition::Zero, shape, st, st,
      axes, levels, y.data(), z.data());
  save(dir + "/host_fwd_" + tag + ".bin", y);
  save(dir + "/host_adj_" + tag + ".bin", z);
  T *dx, *dy, *dz;
  if (cudaMalloc(&dx, n * n * sizeof(T)) || cudaMalloc(&dy, n * n * sizeof(T)) ||
      cudaMalloc(&dz, n * n * sizeof(T)))
    std::exit(12);
  cudaMemcpy(dx, x.data(), n * n * sizeof(T), cudaMemcpyHostToDevice);
  lwt(Wavelet::CDF9_7, Transform::Forward, BoundaryCondition::Zero, shape, st, st, axes,
      levels, dx, dy);
  lwt(Wavelet::CDF9_7, Transform::ForwardAdjoint, BoundaryCondition::Zero, shape, st, st,
      axes, levels, dy, dz);
  // the call returned with the result in place: no synchronisation here
  cudaMemcpy(y.data(), dy, n * n * sizeof(T), cudaMemcpyDeviceToHost);
  cudaMemcpy(z.data(), dz, n * n * sizeof(T), cudaMemcpyDeviceToHost);
  save(dir + "/dev_fwd_" + tag + ".bin", y);
  save(dir + "/dev_adj_" + tag + ".bin", z);
  cudaFree(dx);
  cudaFree(dy);
  cudaFree(dz);
}

// Non-separable (Mallat) 3D transform, 2 levels, Symmetric boundary, on host
// vectors (Forward) and device pointers (Inverse of that result).
template <typename T>
void nonseparable(const std::string& dir, const char* tag) {
  const size_v shape{16, 24, 40}, axes{0, 1, 2};
  const size_t n = 16 * 24 * 40;
  const stride_v st{24 * 40, 40, 1};
  std::vector<T> x = load<T>(dir + "/v_" + tag + ".bin", n), y(n), z(n);
  lwt(Wavelet::Daubechies4, Transform::Forward, BoundaryCondition::Symmetric, shape, st, st,
      axes, size_t{2}, x.data(), y.data());
  save(dir + "/host_nonsep_" + tag + ".bin", y);
  T *dy, *dz;
  if (cudaMalloc(&dy, n * sizeof(T)) || cudaMalloc(&dz, n * sizeof(T))) std::exit(13);
  cudaMemcpy(dy, y.data(), n * sizeof(T), cudaMemcpyHostToDevice);
  lwt(Wavelet::Daubechies4, Transform::Inverse, BoundaryCondition::Symmetric, shape, st, st,
      axes, size_t{2}, dy, dz);
  cudaMemcpy(z.data(), dz, n * sizeof(T), cudaMemcpyDeviceToHost);
  save(dir + "/dev_nonsep_inv_" + tag + ".bin", z);
  cudaFree(dy);
  cudaFree(dz);
}

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  const std::string dir = argv[1];
  separable<float>(dir, "f32");
  separable<double>(dir, "f64");
  nonseparable<float>(dir, "f32");
  nonseparable<double>(dir, "f64");
  std::printf("done\n");
  return 0;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_cpp_overloads_on_host_and_device_pointers(tmp_path):
    src = tmp_path / "dropin.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "dropin"
    lib = _lib.LIB_PATH
    subprocess.run(["g++", "-std=c++20", "-O1", f"-I{ROOT / 'include'}",
                    f"-I{CUDA / 'include'}", str(src), "-o", str(exe), str(lib),
                    f"-L{CUDA / 'lib64'}", "-lcudart", f"-Wl,-rpath,{lib.parent}",
                    f"-Wl,-rpath,{CUDA / 'lib64'}"],
                   check=True, capture_output=True)
    rng = np.random.default_rng(77)
    x = rng.standard_normal((512, 512))
    v = rng.standard_normal((16, 24, 40))
    for tag, dt in (("f32", np.float32), ("f64", np.float64)):
        x.astype(dt).tofile(tmp_path / f"x_{tag}.bin")
        v.astype(dt).tofile(tmp_path / f"v_{tag}.bin")
    r = subprocess.run([str(exe), str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr

    for tag, dt in (("f32", np.float32), ("f64", np.float64)):
        xs = x.astype(dt)
        rc, fwd = po.oracle_sep(xs, 100907, 0, 0, [0, 1], [6, 6])
        assert rc == 0
        rc, adj = po.oracle_sep(fwd, 100907, 2, 0, [0, 1], [6, 6])
        assert rc == 0
        for where in ("host", "dev"):
            got = np.fromfile(tmp_path / f"{where}_fwd_{tag}.bin", dtype=dt).reshape(512, 512)
            assert np.array_equal(got, fwd), (where, tag)
            got = np.fromfile(tmp_path / f"{where}_adj_{tag}.bin", dtype=dt).reshape(512, 512)
            assert np.array_equal(got, adj), (where, tag)
        vs = v.astype(dt)
        rc, nf = po.oracle_nonsep(vs, 4, 0, 3, [0, 1, 2], 2)
        assert rc == 0
        got = np.fromfile(tmp_path / f"host_nonsep_{tag}.bin", dtype=dt).reshape(v.shape)
        assert np.array_equal(got, nf), tag
        rc, ni = po.oracle_nonsep(nf, 4, 1, 3, [0, 1, 2], 2)
        assert rc == 0
        got = np.fromfile(tmp_path / f"dev_nonsep_inv_{tag}.bin", dtype=dt).reshape(v.shape)
        assert np.array_equal(got, ni), tag
