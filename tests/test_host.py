"""Host side of the engine without a GPU: the C ABI loads and exports what
include/lssph.h declares, the config.h surface, particle setup and the results/ format
match the reference restatement bit for bit."""
import ctypes as C
import os
import re
import sys

import numpy as np
import pytest

import lssph
import oracle as O
from lssph import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _header_functions():
    text = open(os.path.join(ROOT, "include", "lssph.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lssph_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = lssph.load()
    declared = _header_functions()
    assert len(declared) >= 30
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) == set(_abi.exported_names())
    assert lib.lssph_abi_version() == 2
    assert lib.lssph_params_sizeof() == C.sizeof(lssph.Params)


def test_default_params_are_the_shipped_config(reference_root):
    p_ref = lssph.from_config(os.path.join(reference_root, "config.h"))
    p_def = lssph.default_params()
    assert p_ref.as_dict() == p_def.as_dict()


def test_config_roundtrip(tmp_path):
    p = lssph.taylor_green_params(num=64, re=250.0, SAVE_NAME="tg_run", end_step=500)
    path = tmp_path / "config.h"
    lssph.write_config_h(p, str(path))
    q = lssph.from_config(str(path))
    assert q.as_dict() == p.as_dict()


def test_config_parser_reads_fortran_literals(tmp_path):
    path = tmp_path / "config.h"
    path.write_text('/* comment */\n#define TARGET_PROBLEM 3\n#define U_BOUNDARY_TOP 3\n#define U_BOUNDARY_BOTTOM 2\n'
                    '#define U_BOUNDARY_LEFT 2\n#define U_BOUNDARY_RIGHT 2\n#define VIS_REF 1.0d-3 /* mu */\n'
                    '#define NUM_X 64\n#define NUM_Y 64\n#define SAVE_NAME "cav"\n')
    p = lssph.from_config(str(path))
    assert p.target_problem == 3 and p.vis_ref == 1.0e-3 and p.num_x == 64
    assert p.save_name == b"cav" and p.dx == 1.0 / 64


@pytest.mark.parametrize("maker", [
    lambda: lssph.default_params(),
    lambda: lssph.diffusion_params(num=50),
    lambda: lssph.taylor_green_params(num=128),
    lambda: lssph.cavity_params(num=256),
    lambda: lssph.boussinesq_params(num=96, ra=1e6),
    lambda: lssph.make_params(KERNEL_TYPE=2, NUM_X=40, NUM_Y=40),
    lambda: lssph.make_params(KERNEL_TYPE=5, COE_H=1.5, ZETA_RSST=2.0, XI_VIM=1.5),
])
def test_init_param_matches_oracle(maker):
    # init_param_mod.f90:92-199, restated twice (engine host + oracle): bit-identical
    p = maker()
    q = O.init_param(p)
    assert p.as_dict() == q.as_dict()


@pytest.mark.parametrize("field,value", [
    ("TARGET_PROBLEM", 5), ("KERNEL_TYPE", 0), ("SPH_MODEL", 7), ("WALL_MODEL", 4), ("RK", 3),
    ("U_BOUNDARY_TOP", 3), ("NUM_X", 0), ("COE_CFL", 1.0), ("ZETA_RSST", 0.5), ("VIS_REF", -1.0),
    ("GRAVITY", -1.0), ("COE_H", 0.0), ("PST_C", -0.1), ("END_STEP", 0), ("TG_A", 0),
])
def test_check_param_rejects_what_the_reference_rejects(field, value):
    # check_param_mod.f90:22-284: every `error stop` is LSSPH_E_BAD_PARAM with a message
    with pytest.raises(lssph.LssphError) as e:
        lssph.make_params(**{field: value})
    assert e.value.status == _abi.E_BAD_PARAM and e.value.message


def test_check_param_isotropic_spacing():
    with pytest.raises(lssph.LssphError, match="isotropic"):
        lssph.make_params(LEN_X=1.0, LEN_Y=1.0, NUM_X=50, NUM_Y=60)


@pytest.mark.parametrize("maker", [
    lambda: lssph.diffusion_params(num=50, seed=5),
    lambda: lssph.taylor_green_params(num=64),
    lambda: lssph.cavity_params(num=40),
    lambda: lssph.boussinesq_params(num=32),
    lambda: lssph.make_params(KERNEL_TYPE=2, NUM_X=30, NUM_Y=30),
])
def test_setup_particles_matches_oracle(maker):
    # setup_closed_box + impose_* restated twice: bit-identical
    p = maker()
    st, ni = lssph.setup_particles(p)
    o = O.Oracle(p, ghost=False)
    g = o.get()
    assert ni == o.num_int and st.num_total == o.num_total
    assert np.array_equal(st.ptype, g["ptype"])
    for k in ("x", "y", "u", "v", "rho", "pre"):
        assert np.array_equal(getattr(st, k), g[k]), k
    if st.tem is not None:
        assert np.array_equal(st.tem, g["tem"])


def test_setup_layout_is_interior_first():
    p = lssph.make_params(NUM_X=50, NUM_Y=50)
    st, ni = lssph.setup_particles(p)
    assert ni == 2500 and st.num_total == 56 * 56
    assert np.all(st.ptype[:ni] == 0) and np.all((st.ptype[ni:] >= 1) & (st.ptype[ni:] <= 8))
    # interior particles in row-major scan order (setup_closed_box_mod.f90:120-136)
    assert np.all(np.diff(st.y[:ni]) >= 0)


def _fortran_e21_14(v):
    if v == 0:
        return " 0.00000000000000E+00"
    s = f"{abs(v):.13E}"
    mant, exp = s.split("E")
    digits = mant.replace(".", "")
    e = int(exp) + 1
    out = ("-" if v < 0 else "") + "0." + digits + ("E%+03d" % e if abs(e) <= 99 else "%+04d" % e)
    return out.rjust(21)


def test_parameters_csv_format(tmp_path):
    # write_param_mod.f90:61-126: `(a, ',', e21.14)` and `(a, ',', i0)` rows
    p = lssph.taylor_green_params(num=128)
    path = tmp_path / "parameters.csv"
    lib = lssph.load()
    assert lib.lssph_write_parameters(C.byref(p), 17956, 16384, str(path).encode()) == 0
    lines = path.read_text().splitlines()
    assert lines[0] == "Parameter, Value"
    rows = dict(line.split(",", 1) for line in lines[1:])
    assert rows["target_problem"] == "2"
    assert rows["num_total"] == "17956" and rows["num_int"] == "16384" and rows["num_ext"] == "1572"
    assert rows["dx"] == " 0.78125000000000E-02"
    assert rows["dt"] == _fortran_e21_14(p.dt)
    assert rows["tem_ave"] == " 0.00000000000000E+00"
    assert len(lines) == 1 + 59    # write_param_mod.f90:64-126: 34 + 22 + 3 rows
    for k, v in rows.items():
        if not re.fullmatch(r"-?\d+", v):
            assert len(v) == 21 and re.fullmatch(r" ?-?0\.\d{14}E[+-]\d\d", v), (k, v)


def test_parameters_csv_reads_with_reference_reader(tmp_path, reference_root):
    sys.path.insert(0, reference_root)
    from analysis.common import read_utils   # the reference's own reader
    p = lssph.boussinesq_params(num=64, ra=1e5)
    path = tmp_path / "parameters.csv"
    assert lssph.load().lssph_write_parameters(C.byref(p), 4900, 4096, str(path).encode()) == 0
    ns = read_utils.parameters(path)
    assert ns.num_int == 4096 and ns.target_problem == 4
    for k in ("dx", "h", "h_eff", "W_ave", "dt", "Ra", "Pr", "thermal_dif", "kinematic_vis"):
        assert getattr(ns, k) == pytest.approx(getattr(p, k), rel=1e-13), k


def test_read_data_reads_stream_layout(tmp_path):
    # restart_mod.f90:32-53 / write_data_mod.f90:40-54: int32 ptype, then float64 fields
    p = lssph.boussinesq_params(num=16)
    st, ni = lssph.setup_particles(p)
    path = tmp_path / "7.dat"
    with open(path, "wb") as f:
        st.ptype.astype("<i4").tofile(f)
        for k in ("x", "y", "u", "v", "rho", "pre", "tem"):
            getattr(st, k).astype("<f8").tofile(f)
    back = lssph.read_data(str(path), p)
    for k in ("ptype", "x", "y", "u", "v", "rho", "pre", "tem"):
        assert np.array_equal(getattr(back, k), getattr(st, k)), k
    with pytest.raises(lssph.LssphError):
        lssph.read_data(str(tmp_path / "missing.dat"), p)


def test_status_strings():
    lib = lssph.load()
    for code in range(0, -11, -1):
        assert lib.lssph_status_string(code)


def test_mixed_precision_runs_two_or_four_lanes():
    # the mixed-precision kernels exist for 2 and 4 lanes per particle; 8 is refused before
    # any device work
    import lssph
    p = lssph.make_params(lssph.taylor_green_params(num=16), precision=lssph.PRECISION_MIXED, lanes=8)
    st, ni = lssph.setup_particles(p)
    with pytest.raises(lssph.LssphError) as e:
        lssph.Simulation(p, st, ni)
    assert e.value.status == lssph._abi.E_UNSUPPORTED


def test_device_footprint_estimate_is_host_only_and_grows_with_size():
    import lssph
    sizes = [lssph.estimate_device_bytes(lssph.taylor_green_params(num=n)) for n in (32, 64, 128)]
    assert 0 < sizes[0] < sizes[1] < sizes[2]
    # FP64 state, RK registers and cell lists: a few hundred bytes per particle
    p = lssph.taylor_green_params(num=128)
    nt, ni = lssph.setup_particles(p)[0].num_total, 128 * 128
    assert 200 * nt < sizes[2] < 2000 * nt


def test_noalloc_rejects_unsupported_options_before_any_gpu_work():
    # lssph_rhs_noalloc checks its options on the host: a periodic domain (its cell grid
    # has no wrap) and lane counts other than 0, 1, 2, 4 return LSSPH_E_UNSUPPORTED with
    # their own messages, before any CUDA call (so this runs without a GPU)
    import ctypes as C

    from lssph import _abi
    lib = lssph.load()
    fake = C.c_void_p(256)   # never dereferenced
    args = lambda n: (n, 1024, *([fake] * 6), None, *([fake] * 3), None, None)   # noqa: E731
    p = lssph.taylor_green_params(num=32, PERIODIC=1)
    assert lib.lssph_rhs_noalloc(C.byref(p), *args(1024)) == _abi.E_UNSUPPORTED
    assert b"closed box only" in lib.lssph_last_error()
    p = lssph.taylor_green_params(num=32, lanes=8)
    assert lib.lssph_rhs_noalloc(C.byref(p), *args(1444)) == _abi.E_UNSUPPORTED
    assert b"lanes must be" in lib.lssph_last_error()
    p = lssph.taylor_green_params(num=32)
    assert lib.lssph_rhs_noalloc(C.byref(p), *args(262145)) == _abi.E_CAPACITY


def test_mapped_downloads_need_device_write_access(tmp_path):
    # the predicate that keeps k_download_mapped away from page-locked buffers the device may
    # only read (cudaHostRegisterReadOnly): only read-write access flags allow the in-place
    # kernel; read-only, none and "driver could not say" (-1) go through copies
    import subprocess
    hdr = os.path.join(os.path.dirname(lssph.__file__), "..", "csrc", "hostmem.h")
    src = tmp_path / "t.cpp"
    src.write_text('#include "%s"\n#include <cstdio>\nint main() { const long long fl[] = {-1, 0, 1, 2, 3}; for (long long f : fl)'
                   ' std::printf("%%lld:%%d ", f, (int)lssph::mapped_store_allowed(f)); }\n' % hdr)
    exe = tmp_path / "t"
    subprocess.run(["g++", "-std=c++17", str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    assert out == ["-1:0", "0:0", "1:0", "2:0", "3:1"]
