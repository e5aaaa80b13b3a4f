"""The C ABI from C: include/duvi_gpu.h compiles as C99 with every warning an error,
and a C program linked against libduvigpu.so runs the host-side entry points end to
end (a hex operator, both DuVi encoders, the Unit stream round trip) and gets the
no-device status from dv_context_create on a machine without a GPU.  This is the
surface a P/Invoke, cgo or JNI binding sees."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "..")

PROGRAM = r"""
#include "duvi_gpu.h"
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define CHECK(x) do { int s_ = (x); if (s_ != DV_OK) { \
    printf("fail %s: %d %s\n", #x, s_, dv_last_error()); return 1; } } while (0)

int main(void) {
    const int32_t ne[3] = {3, 2, 2};
    int32_t n = 0;
    int64_t nnz = 0;
    CHECK(dv_hex_csr_size(ne, &n, &nnz));
    int32_t *rp = malloc(sizeof(int32_t) * (size_t)(n + 1));
    int32_t *ci = malloc(sizeof(int32_t) * (size_t)nnz);
    double *va = malloc(sizeof(double) * (size_t)nnz);
    CHECK(dv_hex_assemble(ne, NULL, 1.0, 1.0, 0.3, rp, ci, va));
    dv_csr_host a;
    a.n_rows = n; a.n_cols = n; a.rowptr = rp; a.col = ci; a.val = va;

    int64_t nb = 0, nu = 0;
    int32_t bits = 0;
    CHECK(dv_duvi_encode(&a, 0, 1e-10, &nb, &nu, &bits, NULL, NULL, NULL, NULL, NULL, NULL));
    uint32_t *r2c = malloc(sizeof(uint32_t) * (size_t)(n + 1)), *r2d = malloc(sizeof(uint32_t) * (size_t)(n + 1));
    uint32_t *cidx = malloc(sizeof(uint32_t) * (size_t)nb), *vidx = malloc(sizeof(uint32_t) * (size_t)nnz);
    uint8_t *dist = malloc((size_t)nnz);
    double *vals = malloc(sizeof(double) * (size_t)nu);
    CHECK(dv_duvi_encode(&a, 0, 1e-10, &nb, &nu, &bits, r2c, r2d, cidx, dist, vidx, vals));

    int64_t n_units = 0, n_bytes = 0, n_idx = 0, nq = 0;
    CHECK(dv_units_encode(&a, 1e-10, &n_units, &n_bytes, &n_idx, &nq, NULL, NULL, NULL, NULL));
    uint8_t *ub = malloc((size_t)n_bytes);
    int64_t *uo = malloc(sizeof(int64_t) * (size_t)(n_units + 1));
    int32_t *ui = malloc(sizeof(int32_t) * (size_t)n_idx);
    double *uv = malloc(sizeof(double) * (size_t)nq);
    CHECK(dv_units_encode(&a, 1e-10, &n_units, &n_bytes, &n_idx, &nq, ub, uo, ui, uv));
    int64_t nnz2 = 0;
    CHECK(dv_units_decode(n, n, ub, n_bytes, ui, n_idx, uv, nq, &nnz2, NULL, NULL, NULL));
    int32_t *rp2 = malloc(sizeof(int32_t) * (size_t)(n + 1)), *ci2 = malloc(sizeof(int32_t) * (size_t)nnz2);
    double *va2 = malloc(sizeof(double) * (size_t)nnz2);
    CHECK(dv_units_decode(n, n, ub, n_bytes, ui, n_idx, uv, nq, &nnz2, rp2, ci2, va2));
    if (nnz2 != nnz || memcmp(rp, rp2, sizeof(int32_t) * (size_t)(n + 1)) != 0 ||
        memcmp(ci, ci2, sizeof(int32_t) * (size_t)nnz) != 0 || memcmp(va, va2, sizeof(double) * (size_t)nnz) != 0) {
        printf("fail: unit round trip differs\n");
        return 1;
    }

    dv_context *ctx = NULL;
    int st = dv_context_create(0, &ctx);
    if (st == DV_OK) dv_context_destroy(ctx);
    printf("ok n=%d nnz=%lld nblocks=%lld nuniq=%lld bits=%d units=%lld bytes=%lld context=%s\n", n,
           (long long)nnz, (long long)nb, (long long)nu, bits, (long long)n_units, (long long)n_bytes,
           dv_status_string(st));
    return (st == DV_OK || st == DV_ERR_NO_DEVICE) ? 0 : 1;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_header_compiles_as_c_and_host_entry_points_run(tmp_path, native):
    src = tmp_path / "abi.c"
    src.write_text(PROGRAM)
    exe = tmp_path / "abi"
    lib_dir = os.path.join(ROOT, "compressiontests_b200")
    cmd = ["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", os.path.join(ROOT, "include"),
           str(src), "-o", str(exe), "-L", lib_dir, "-lduvigpu", f"-Wl,-rpath,{lib_dir}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    # the library's own dependencies (the CUDA runtime) resolve from where this process loaded them
    env = dict(os.environ)
    cudart = [p for p in open("/proc/self/maps").read().split() if "libcudart.so" in p]
    if cudart:
        env["LD_LIBRARY_PATH"] = os.path.dirname(cudart[0]) + ":" + env.get("LD_LIBRARY_PATH", "")
    r = subprocess.run([str(exe)], capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("ok "), r.stdout
    print(r.stdout.strip())
