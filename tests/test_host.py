"""Host-side logic of the product, no GPU: the C ABI library loads and
exports every declared symbol, and its header compiles as strict C and links
from a C program; the FP64 cosmology, COLA coefficients and
P(k) spline agree with the oracle; the draw generator is uniform and keyed by
mode; the Python package imports; argument errors map to the reference's
exceptions."""
import ctypes as C
import math
import os

import numpy as np
import pytest

from fs2_b200 import capi


def test_library_exports_every_header_symbol():
    lib = capi.lib()
    names = capi.header_functions()
    assert len(names) > 60
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the binding covers the whole header
    assert sorted(capi._SIGS) == names


def test_fs_package_imports():
    import fs2_b200.fs as fs
    assert fs.comm.this_node() == 0 and fs.comm.n_nodes() == 1
    assert fs.config_precision() == "single"
    for name in ("init", "force", "send_positions", "compute_density",
                 "check_total_density", "compute_force", "get_forces"):
        assert callable(getattr(fs.pm, name))
    assert callable(fs.cola.kick) and callable(fs.cola.drift)
    assert callable(fs.lpt.init)


def _d(fn, *args):
    out = C.c_double()
    capi.call(fn, *args, C.byref(out))
    return out.value


def test_cosmology_matches_oracle(oracle_mod):
    capi.call("fs2g_cosmology_init", 0.31)
    o = oracle_mod.Cosmology(0.31)
    for a in (0.02, 0.1, 0.25, 0.5, 0.75, 1.0):
        D = _d("fs2g_cosmology_D_growth", a)
        assert D == pytest.approx(o.D(a), rel=1e-12)
        assert _d("fs2g_cosmology_D2_growth", a, D) == pytest.approx(
            o.D2(a, D), rel=1e-12)
        assert _d("fs2g_cosmology_f_growth_rate", a) == pytest.approx(
            o.f(a), rel=1e-10)
        assert _d("fs2g_cosmology_Dv_growth", a, D) == pytest.approx(
            o.Dv(a, D), rel=1e-10)
        assert _d("fs2g_cosmology_hubble_function", a) == pytest.approx(
            o.hubble(a), rel=1e-15)
    assert _d("fs2g_cosmology_D_growth", 0.0) == 0.0


def test_cosmology_einstein_de_sitter_known_answers():
    # Omega_m = 1: H = a^(-3/2), so D = a, f = 1 and the second-order growth
    # D2 = -3/7 D^2 Omega^(-1/143) = -3/7 a^2 (py/cosmology.cpp:24-66)
    try:
        capi.call("fs2g_cosmology_init", 1.0)
        assert _d("fs2g_cosmology_D_growth", 1.0) == pytest.approx(1.0,
                                                                   abs=1e-14)
        for a in (0.02, 0.1, 0.5, 1.0):
            D = _d("fs2g_cosmology_D_growth", a)
            assert D == pytest.approx(a, rel=1e-12)
            assert _d("fs2g_cosmology_f_growth_rate", a) == pytest.approx(
                1.0, rel=1e-10)
            assert _d("fs2g_cosmology_D2_growth", a, D) == pytest.approx(
                -3.0 / 7.0 * a * a, rel=1e-12)
            assert _d("fs2g_cosmology_hubble_function", a) == pytest.approx(
                a ** -1.5, rel=1e-14)
    finally:
        capi.call("fs2g_cosmology_init", 0.31)


def test_cola_coefficients_match_oracle(oracle_mod):
    capi.call("fs2g_cosmology_init", 0.31)
    cosmo = oracle_mod.Cosmology(0.31)
    a_v, a_x = 0.1, 0.1
    for a_vel, a_pos in ((0.145, 0.19), (0.55, 0.6), (0.955, 1.0)):
        om, kf, q1, q2 = C.c_double(), C.c_float(), C.c_float(), C.c_float()
        capi.call("fs2g_cola_kick_coef", a_v, a_x, a_vel, C.byref(om),
                  C.byref(kf), C.byref(q1), C.byref(q2))
        r = oracle_mod.kick_coefficients(cosmo, a_v, a_x, a_vel)
        assert om.value == pytest.approx(-1.5 * r[0], rel=1e-15)
        # Float results: equal after rounding, or one ulp apart at a tie
        for got, want in ((kf.value, r[1]), (q1.value, r[2]), (q2.value, r[3])):
            assert np.float32(got) == pytest.approx(want, rel=1.2e-7)
        dt, da1, da2 = C.c_double(), C.c_float(), C.c_float()
        capi.call("fs2g_cola_drift_coef", a_x, a_vel, a_pos, C.byref(dt),
                  C.byref(da1), C.byref(da2))
        d = oracle_mod.drift_coefficients(cosmo, a_x, a_vel, a_pos)
        assert dt.value == pytest.approx(d[0], rel=1e-12)
        assert np.float32(da1.value) == pytest.approx(d[1], rel=1.2e-7)
        assert np.float32(da2.value) == pytest.approx(d[2], rel=1.2e-7)
        a_v, a_x = a_vel, a_pos


def test_power_spectrum_matches_oracle(oracle_mod, eh_table):
    ps = C.c_void_p()
    capi.call("fs2g_power_alloc", eh_table.encode(), C.byref(ps))
    try:
        o = oracle_mod.PowerSpectrum(eh_table)
        n = C.c_int()
        capi.call("fs2g_power_n", ps, C.byref(n))
        assert n.value == o.n == 1000
        for k in np.logspace(-3.5, 2.5, 37):
            assert _d("fs2g_power_P", ps, float(k)) == pytest.approx(
                float(o.P(k)), rel=1e-11)
        assert _d("fs2g_power_sigma", ps, 8.0) == pytest.approx(0.81,
                                                                rel=1e-12)
        k, P = C.c_double(), C.c_double()
        capi.call("fs2g_power_i", ps, 0, C.byref(k), C.byref(P))
        assert k.value == pytest.approx(1e-4)
        assert capi.lib().fs2g_power_i(ps, 1000, C.byref(k), C.byref(P)) == -8
        # outside the table: a domain error, as GSL's interpolation gives
        assert capi.lib().fs2g_power_P(ps, 1e4, C.byref(P)) == -5
    finally:
        capi.lib().fs2g_power_free(ps)


def test_power_file_errors(tmp_path):
    ps = C.c_void_p()
    rc = capi.lib().fs2g_power_alloc(str(tmp_path / "missing").encode(),
                                     C.byref(ps))
    assert rc == -3                                        # IOError
    bad = tmp_path / "unsorted.dat"
    bad.write_text("# k P\n0.1 10\n0.01 20\n1.0 5\n")
    assert capi.lib().fs2g_power_alloc(str(bad).encode(), C.byref(ps)) == -3
    ok = tmp_path / "ok.dat"
    # comment lines, a k <= 0 row skipped, reading stops at a bad line
    ok.write_text("# header\n-1 3\n0.01 20\n0.1 10\n1.0 5\nnot numbers\n9 9\n")
    capi.call("fs2g_power_alloc", str(ok).encode(), C.byref(ps))
    n = C.c_int()
    capi.call("fs2g_power_n", ps, C.byref(n))
    assert n.value == 3
    capi.lib().fs2g_power_free(ps)


def test_python_power_spectrum_api(eh_table):
    import fs2_b200.fs as fs
    ps = fs.PowerSpectrum(eh_table)
    assert len(ps) == 1000
    k, P = ps[10]
    assert k > 0 and P > 0
    with pytest.raises(IndexError):
        ps[1000]
    with pytest.raises(IOError):
        fs.PowerSpectrum("/nonexistent/pk.dat")


def test_lpt_draws_uniform_and_keyed_by_mode():
    import fs2_b200.fs as fs
    up, ua = fs.lpt.draws(32, 11)
    assert up.shape == (32, 32, 16)
    for u in (up, ua):
        assert u.min() > 0.0 and u.max() < 1.0
        assert abs(u.mean() - 0.5) < 0.01
        assert abs(u.var() - 1.0 / 12) < 0.005
    assert abs(np.corrcoef(up.ravel(), ua.ravel())[0, 1]) < 0.02
    # same seed -> same draws; another seed -> others
    up2, _ = fs.lpt.draws(32, 11)
    assert np.array_equal(up, up2)
    assert not np.array_equal(up, fs.lpt.draws(32, 12)[0])
    # a mode keeps its draws at any nc that holds it (signed kx, ky keys)
    small, _ = fs.lpt.draws(16, 11)
    for kx in (-7, -1, 0, 3, 7):
        for ky in (-5, 0, 6):
            ix16, iy16 = kx % 16, ky % 16
            ix32, iy32 = kx % 32, ky % 32
            assert np.array_equal(small[ix16, iy16, :7], up[ix32, iy32, :7])


def test_eh_table_normalisation():
    from fs2_b200 import power_eh
    k, P = power_eh.eh_nowiggle_table()
    assert power_eh.sigma_trapezoid(k, P, 8.0) == pytest.approx(0.81)
    assert np.all(P > 0) and np.all(np.diff(k) > 0)
    # the EH98 no-wiggle T(k) -> 1 on large scales
    T = power_eh.transfer_nowiggle(np.array([1e-5]), 0.31, 0.049, 0.67)
    assert T[0] == pytest.approx(1.0, abs=1e-3)


def test_capsule_type_errors():
    import fs2_b200.fs as fs
    with pytest.raises(TypeError):
        fs._fs._particles_len(object())
    with pytest.raises(TypeError):
        fs.cola.kick(type("P", (), {"_particles": object()})(), 0.5)


def test_snapshot_datasets_layout():
    # save_hdf5's datasets for an option string (py/hdf5_write.cpp:28-187),
    # with a stand-in particle set so that no GPU is needed
    import numpy as np
    import pytest
    import fs2_b200.fs as fs
    from fs2_b200.fs.particles import snapshot_datasets

    class Stub:
        a = (0.5, 0.45, 0.5)
        boxsize = 64.0
        np_total = 27
        id = np.arange(1, 28, dtype=np.uint64)
        x = np.ones((27, 3), np.float32)
        v = 2 * x
        force = 3 * x
        dx1 = 4 * x
        dx2 = 5 * x

    fs.cosmology.init(0.31)
    d = snapshot_datasets(Stub(), "ixvf12")
    assert sorted(k for k in d if not k.startswith("parameters/")) == \
        ["dx1", "dx2", "f", "id", "v", "x"]
    assert float(d["parameters/omega_m"]) == 0.31
    assert int(d["parameters/nc"]) == 3 and d["parameters/nc"].dtype == np.int32
    assert float(d["parameters/ax"]) == 0.5 and float(d["parameters/av"]) == 0.45
    assert np.array_equal(d["f"], Stub.force)
    assert sorted(snapshot_datasets(Stub(), "x2")) == \
        ["dx2", "parameters/av", "parameters/ax", "parameters/boxsize",
         "parameters/nc", "parameters/omega_m", "x"]
    with pytest.raises(ValueError):
        snapshot_datasets(Stub(), "xi")          # out of order
    with pytest.raises(ValueError):
        snapshot_datasets(Stub(), "q")


def test_fused_pass_probe_rejects_bad_arguments():
    # argument checks happen before any device call
    import ctypes as C
    from fs2_b200 import capi
    ms = C.c_double()
    for args in ((5, 32, 1), (-1, 32, 1), (0, 0, 1), (0, 2048, 1), (2, 16, 1),
                 (1, 32, 0)):
        with pytest.raises(capi.FS2GError):
            capi.call("fs2g_fused_pass_probe", *args, C.byref(ms))


def test_workload_draws_match_the_library():
    # the numpy restatement of the draw generator (used by the benchmark's
    # CPU reference arm, which must not run the library) gives the library's
    # draws bit for bit
    import fs2_b200.fs as fs
    from fs2_b200 import workloads
    for nc, seed in ((8, 1), (16, 42), (32, 7)):
        a = workloads.lpt_draws(nc, seed)
        b = fs.lpt.draws(nc, seed)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_header_is_plain_c_and_links(tmp_path):
    # include/fs2gpu.h is the boundary for C callers (the reference's C++
    # core, cgo, any FFI): it must compile as strict C99 and as C++17, and a
    # C program must link against libfs2gpu and call its host functions
    import shutil
    import subprocess
    cc = shutil.which("gcc")
    cxx = shutil.which("g++")
    if cc is None or cxx is None:
        pytest.skip("no host compiler")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    inc = os.path.join(root, "include")
    libdir = os.path.dirname(capi.lib()._name)
    src = tmp_path / "use.c"
    src.write_text(
        '#include <stdio.h>\n#include "fs2gpu.h"\n'
        "int main(void) {\n"
        "  double D = 0.0;\n"
        "  if(fs2g_stage_count() <= 0) return 1;\n"
        "  if(fs2g_cosmology_init(1.0) != FS2G_OK) return 2;\n"
        "  if(fs2g_cosmology_D_growth(0.5, &D) != FS2G_OK) return 3;\n"
        "  if(D < 0.4999999 || D > 0.5000001) return 4;\n"
        "  if(fs2g_cosmology_init(-1.0) == FS2G_OK) return 5;\n"
        "  if(fs2g_last_error()[0] == 0) return 6;\n"
        '  printf("%d %.9f\\n", fs2g_version(), D);\n'
        "  return 0;\n}\n")
    exe = tmp_path / "use"
    subprocess.run([cc, "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic",
                    "-I", inc, str(src), "-o", str(exe), "-L", libdir,
                    "-lfs2gpu", "-Wl,-rpath," + libdir], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, (out.returncode, out.stderr)
    assert out.stdout.split()[1] == "0.500000000"
    cpp = tmp_path / "use.cpp"
    cpp.write_text('#include "fs2gpu.h"\nint main() { return fs2g_version() > 0 ? 0 : 1; }\n')
    subprocess.run([cxx, "-std=c++17", "-Wall", "-Werror", "-I", inc,
                    str(cpp), "-o", str(tmp_path / "usecpp"), "-L", libdir,
                    "-lfs2gpu", "-Wl,-rpath," + libdir], check=True)
