"""CPU tests of the C-ABI library: it loads, and exports every entry point
include/rpa_b200.h declares.  No compute call is made without a GPU."""
import ctypes

import numpy as np

import pytest


def test_library_exports_every_declared_symbol(pkg):
    lib = pkg.load_library()
    names = pkg.declared_functions()
    assert "rpa_b200_ec" in names and "rpa_b200_pi" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings(pkg):
    lib = pkg.load_library()
    assert lib.rpa_b200_status_string(pkg.RPA_OK) == b"success"
    assert b"positive definite" in lib.rpa_b200_status_string(pkg.RPA_ERR_NOT_SPD)
    assert lib.rpa_b200_status_string(999) == b"unknown status"


def test_library_exports_nothing_but_the_declared_api(pkg):
    # hidden default visibility: the only exported functions are the rpa_b200_* entry points
    import shutil
    import subprocess
    nm = shutil.which("nm")
    if nm is None:
        pytest.skip("nm not available")
    out = subprocess.run([nm, "-D", "--defined-only", str(pkg.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    funcs = {line.split()[-1] for line in out.splitlines() if len(line.split()) == 3 and line.split()[1] in "TtWi"}
    assert funcs == set(pkg.declared_functions()), sorted(funcs ^ set(pkg.declared_functions()))


def test_ctypes_signatures_match_the_header(pkg):
    # every binding's argtypes agree with the prototype in include/rpa_b200.h: same count, and
    # int64_t -> c_int64, uint64_t -> c_uint64, double -> c_double, int -> c_int, pointer -> pointer
    import re
    text = re.sub(r"/\*.*?\*/", " ", pkg.HEADER.read_text(), flags=re.S)
    lib = pkg.load_library()
    checked = 0
    for m in re.finditer(r"^\s*(?:int64_t|int|const char\*)\s+(rpa_b200_\w+)\s*\(([^;]*?)\)\s*;", text, re.M):
        name, params = m.group(1), " ".join(m.group(2).split())
        params = [] if params in ("", "void") else [p.strip() for p in params.split(",")]
        argtypes = getattr(lib, name).argtypes
        assert argtypes is not None and len(argtypes) == len(params), name
        for p, t in zip(params, argtypes):
            if "*" in p:
                assert t is ctypes.c_void_p or issubclass(t, (ctypes._Pointer, ctypes.c_char_p)), (name, p, t)
            elif p.startswith("uint64_t"):
                assert t is ctypes.c_uint64, (name, p, t)
            elif p.startswith("int64_t"):
                assert t is ctypes.c_int64, (name, p, t)
            elif p.startswith("double"):
                assert t is ctypes.c_double, (name, p, t)
            elif p.startswith("int "):
                assert t is ctypes.c_int, (name, p, t)
            else:
                raise AssertionError(f"{name}: unhandled parameter type {p!r}")
        checked += 1
    assert checked == len(pkg.declared_functions())


def test_fortran_interfaces_cover_the_header(pkg):
    # every C entry point has a bind(C) interface in the Fortran module include/rpa_b200_iface.f90,
    # with as many dummy arguments as the prototype has parameters
    import re
    header = re.sub(r"/\*.*?\*/", " ", pkg.HEADER.read_text(), flags=re.S)
    protos = {m.group(1): [p for p in " ".join(m.group(2).split()).split(",") if p.strip() not in ("", "void")]
              for m in re.finditer(r"^\s*(?:int64_t|int|const char\*)\s+(rpa_b200_\w+)\s*\(([^;]*?)\)\s*;",
                                   header, re.M)}
    doc = (pkg.HEADER.parent / "rpa_b200_iface.f90").read_text()
    doc = re.sub(r"&\s*\n\s*", " ", doc)  # join Fortran continuation lines
    binds = {m.group(3): [a for a in m.group(2).split(",") if a.strip()]
             for m in re.finditer(r"function\s+(\w+)\s*\(([^)]*)\)\s*bind\(C,\s*name=\"(\w+)\"\)", doc)}
    assert set(protos) <= set(binds), sorted(set(protos) - set(binds))
    for name, params in protos.items():
        assert len(binds[name]) == len(params), (name, binds[name], params)


def test_plain_c_caller(pkg, tmp_path):
    # the header is valid C99 and the library links and runs from a C program
    import shutil
    import subprocess
    import torch
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    libdir = pkg.LIB_PATH.parent
    exe = tmp_path / "c_abi_harness"
    src = pkg.HEADER.parents[1] / "tests" / "c_abi_harness.c"
    subprocess.run([cc, "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", f"-I{pkg.HEADER.parent}", str(src),
                    f"-L{libdir}", "-lrpa_b200", f"-Wl,-rpath,{libdir}", "-lm", "-o", str(exe)], check=True)
    args = [str(exe)] + ([] if torch.cuda.is_available() else ["nogpu"])
    out = subprocess.run(args, capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stderr


def test_status_codes_match_the_header(pkg):
    import re
    text = pkg.HEADER.read_text()
    enum = dict((m.group(1), int(m.group(2))) for m in re.finditer(r"\b(RPA_(?:OK|ERR_\w+))\s*=\s*(\d+)", text))
    assert enum["RPA_ERR_INTERNAL"] == 10
    for name, value in enum.items():
        assert getattr(pkg, name) == value, name
    lib = pkg.load_library()
    strings = [lib.rpa_b200_status_string(v) for v in sorted(enum.values())]
    assert b"unknown status" not in strings and len(set(strings)) == len(strings)


def test_no_entry_point_lets_an_exception_escape(pkg):
    # every exported int-returning definition is a function-try-block with a catch-all handler
    import re
    csrc = pkg.HEADER.parents[1] / "beyond-rpa_b200" / "csrc"
    seen = 0
    for path in sorted(csrc.glob("*.cu")):
        src = path.read_text()
        for m in re.finditer(r'^(?:extern "C" )?int (rpa_b200_\w+)\(', src, re.M):
            brace = src.index("{", m.end())
            assert src[:brace].endswith(") try "), f"{path.name}: {m.group(1)} is not a function-try-block"
            close = src.index("\n}", brace)
            assert src.startswith("\n} catch (...) {", close), f"{path.name}: {m.group(1)} has no catch-all"
            seen += 1
    declared = [n for n in pkg.declared_functions() if n not in
                ("rpa_b200_status_string", "rpa_b200_last_error", "rpa_b200_last_launches")]
    assert seen == len(declared)


def test_create_without_gpu_reports_no_device(pkg):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    lib = pkg.load_library()
    h = ctypes.c_void_p()
    assert lib.rpa_b200_create(ctypes.byref(h), 0, 0) == pkg.RPA_ERR_NO_DEVICE
    assert not h.value
    with pytest.raises(pkg.RPAError):
        pkg.Handle(0)


def test_null_handle_is_rejected(pkg):
    lib = pkg.load_library()
    assert lib.rpa_b200_destroy(None) == pkg.RPA_OK
    assert lib.rpa_b200_ec_from_pi(None, 4, 1, None, 4, None, None, None) == pkg.RPA_ERR_INVALID_ARG


def test_freq_grid_matches_oracle(pkg, oracle):
    # host-side grid generator of the library vs the oracle restatement
    s = oracle.make_system(10, 12, 150, 5, occ_range=(-1.2, -0.3), virt_range=(0.02, 5.0), ncore_orbs=2)
    core = np.array([-20.3, -19.7])
    e = np.concatenate([core, s.eps_o, s.eps_v])
    for nfixed in (12, 16):
        x, w = pkg.freq_grid(e, len(core) + s.no, s.nv, nfixed=nfixed)
        xr, wr = oracle.grid_for(s, nfixed)
        assert np.allclose(x, xr, rtol=1e-12) and np.allclose(w, wr, rtol=1e-12)
    x, w = pkg.freq_grid(e, len(core) + s.no, s.nv)
    xr, wr = oracle.grid_for(s)
    assert len(x) == len(xr) and np.allclose(x, xr, rtol=1e-12)


@pytest.mark.parametrize("seed,no,nv,occ,virt", [
    (11, 1, 1, (-0.6, -0.5), (0.2, 0.3)),      # one excitation: every histogram bin but one empty
    (12, 3, 40, (-0.4, -0.35), (0.01, 0.05)),  # small gap, narrow spread
    (13, 30, 400, (-2.5, -0.2), (0.05, 60.0)),  # wide spread of excitation energies
    (14, 7, 7, (-1.0, -0.9), (2.0, 2.1)),      # large gap, near-degenerate levels
])
def test_freq_grid_matches_oracle_on_varied_spectra(pkg, oracle, seed, no, nv, occ, virt):
    # Where the best grid of n points still has a quadrature error above rounding, the optimum
    # scale is unique and the library's grid equals the oracle's.  Where n points integrate every
    # 1/(D^2 + u^2) to rounding level (many points, narrow spectra), the error is flat in the
    # scale and its argmin is decided by rounding noise, which differs between implementations
    # (the reference's included): there the library's grid must reach rounding level too.
    import math
    s = oracle.make_system(4, no, nv, seed, occ_range=occ, virt_range=virt)
    e = np.concatenate([s.eps_o, s.eps_v])
    d = (s.eps_v[:, None] - s.eps_o[None, :]).ravel()

    def quad_error(x, w):
        exact = math.pi / (2.0 * d)
        return float(np.max(np.abs(np.sum(w[None, :] / (d[:, None] ** 2 + x[None, :] ** 2), axis=1) - exact) / exact))

    for nfixed in (8, 20, 64, None):
        x, w = pkg.freq_grid(e, no, nv, nfixed=nfixed or 0)
        xr, wr = oracle.grid_for(s, nfixed)
        assert len(x) == len(xr) and (nfixed is None or len(x) == nfixed)
        if quad_error(xr, wr) > 1e-12:
            assert np.allclose(x, xr, rtol=1e-12) and np.allclose(w, wr, rtol=1e-12)
        else:
            assert quad_error(x, w) < 1e-13


def test_freq_grid_unreachable_target_is_reported(pkg, oracle):
    # no grid of up to 64 points meets the targets: the reference stops with "Quadrature did not
    # converge to specified accuracy" (rpa_OptimizeFreqQuad); the library returns a status
    s = oracle.make_system(4, 5, 30, 3, occ_range=(-1.0, -0.3), virt_range=(0.05, 3.0))
    e = np.concatenate([s.eps_o, s.eps_v])
    with pytest.raises(pkg.RPAError) as err:
        pkg.freq_grid(e, 5, 30, target_error=1e-30, target_rel_error=1e-30)
    assert err.value.status == pkg.RPA_ERR_NOT_CONVERGED
    vals, wts = oracle.dai_histogram(e, 5, 30)
    with pytest.raises(RuntimeError):
        oracle.optimize_freq_quad(vals, wts, target_error=1e-30, target_rel_error=1e-30)


def test_freq_grid_rejects_bad_gap(pkg):
    e = np.array([-1.0, 0.5, 0.2, 1.0])  # HOMO above LUMO
    with pytest.raises(pkg.RPAError):
        pkg.freq_grid(e, 2, 2)


def test_plan_entry_points_reject_a_null_handle(pkg):
    lib = pkg.load_library()
    assert lib.rpa_b200_tune_logdet(None, 512, 4, None, None, None) == pkg.RPA_ERR_INVALID_ARG
    assert lib.rpa_b200_set_logdet_plan(None, 512, 256, 64) == pkg.RPA_ERR_INVALID_ARG
    assert lib.rpa_b200_get_logdet_plan(None, 512, None, None) == pkg.RPA_ERR_INVALID_ARG
    assert lib.rpa_b200_set_autotune(None, 1) == pkg.RPA_ERR_INVALID_ARG


@pytest.mark.parametrize("nbody", [2, 3, 4])
def test_mbe_energy_matches_oracle(pkg, oracle, nbody):
    # host entry point: interaction / nonadditive energies from subsystem energies of ~-100 Eh
    rng = np.random.default_rng(40 + nbody)
    for _ in range(50):
        e = -100.0 * rng.uniform(0.5, 2.0, 15)
        e[0] = np.sum(e[1:4]) + rng.uniform(-1e-2, 1e-2)  # a whole system near its parts
        got = pkg.mbe_energy(e, nbody)
        assert got == oracle.mbe_energy(nbody, e)


def test_mbe_energy_of_additive_subsystems_vanishes(pkg):
    # exactly additive energies (sums of monomers) give zero interaction at every order
    a, b, c, d = -76.123456789012345, -40.5, -0.25, -12.0009765625
    e = [a + b + c + d, a, b, c, a + b, b + c, a + c, d, a + d, b + d, c + d,
         a + b + c, a + b + d, a + c + d, b + c + d]
    assert abs(pkg.mbe_energy([a + b, a, b], 2)) <= 1e-14
    e3 = [a + b + c] + e[1:7]
    assert abs(pkg.mbe_energy(e3, 3)) <= 1e-13
    assert abs(pkg.mbe_energy(e, 4)) <= 1e-13


def test_mbe_energy_rejects_bad_arguments(pkg):
    lib = pkg.load_library()
    assert lib.rpa_b200_mbe_energy(5, None, None) == pkg.RPA_ERR_INVALID_ARG
    with pytest.raises(ValueError):
        pkg.mbe_energy([1.0, 2.0], 3)


def _cluster_sets(seed=7):
    # a dimer AB and its monomers in the dimer basis: the monomers carry ghost virtuals far above
    # the complex's highest excitation, which the capped histograms must ignore
    rng = np.random.default_rng(seed)
    def orbitals(nocc, nvirt, ghosts):
        occ = np.sort(np.concatenate([[-20.3], rng.uniform(-1.3, -0.4, nocc - 1)]))
        virt = np.sort(np.concatenate([np.exp(rng.uniform(np.log(0.03), np.log(4.0), nvirt)),
                                       rng.uniform(8.0, 40.0, ghosts)]))
        return occ, virt
    oa, va = orbitals(4, 30, 6)
    ob, vb = orbitals(3, 26, 8)
    oab = np.sort(np.concatenate([oa, ob]))
    vab = np.sort(np.concatenate([va[va < 5.0], vb[vb < 5.0]]))
    return [(np.concatenate([oab, vab]), len(oab), len(vab)),
            (np.concatenate([oa, va]), len(oa), len(va)),
            (np.concatenate([ob, vb]), len(ob), len(vb))]


@pytest.mark.parametrize("limit", [True, False])
def test_freq_grid_mbe_matches_oracle(pkg, oracle, limit):
    sets = _cluster_sets()
    x, w = pkg.freq_grid_mbe(sets, limit_dai=limit, nfixed=12)
    xr, wr = oracle.grid_for_cluster(sets, limit_dai=limit, n=12)
    assert np.allclose(x, xr, rtol=1e-12) and np.allclose(w, wr, rtol=1e-12)
    x, w = pkg.freq_grid_mbe(sets, limit_dai=limit)
    xr, wr = oracle.grid_for_cluster(sets, limit_dai=limit)
    assert len(x) == len(xr) and np.allclose(x, xr, rtol=1e-12) and np.allclose(w, wr, rtol=1e-12)


def test_freq_grid_mbe_of_one_set_is_the_single_grid(pkg):
    (e, no, nv), = _cluster_sets()[:1]
    x1, w1 = pkg.freq_grid(e, no, nv, nfixed=10)
    x2, w2 = pkg.freq_grid_mbe([(e, no, nv)], nfixed=10)
    assert np.array_equal(x1, x2) and np.array_equal(w1, w2)


def test_freq_grid_mbe_set_above_the_cap_takes_no_part(pkg, oracle):
    # a subsystem whose smallest excitation energy lies above the complex's largest one has no
    # difference under the cap (its histogram weights are 0/0, as in the reference) and leaves
    # the capped grid unchanged; without the cap it counts
    sets = _cluster_sets()
    cap = oracle.dai_max_thresh(*sets[0])  # the complex's largest active excitation energy
    far = (np.array([-0.5, -0.4, cap + 0.1, cap + 0.3]), 2, 2)
    x1, w1 = pkg.freq_grid_mbe(sets, nfixed=10)
    x2, w2 = pkg.freq_grid_mbe(sets + [far], nfixed=10)
    assert np.array_equal(x1, x2) and np.array_equal(w1, w2)
    xr, wr = oracle.grid_for_cluster(sets + [far], limit_dai=True, n=10)
    assert np.allclose(x2, xr, rtol=1e-12) and np.allclose(w2, wr, rtol=1e-12)
    x3, _ = pkg.freq_grid_mbe(sets + [far], limit_dai=False, nfixed=10)
    xr3, _ = oracle.grid_for_cluster(sets + [far], limit_dai=False, n=10)
    assert np.allclose(x3, xr3, rtol=1e-12)


def test_freq_grid_mbe_skips_all_core_sets_and_rejects_bad_gaps(pkg):
    sets = _cluster_sets()
    core_only = (np.array([-25.0, -21.0, 0.5, 1.0, 2.0]), 2, 3)  # every occupied orbital frozen
    x1, _ = pkg.freq_grid_mbe(sets, nfixed=10)
    x2, _ = pkg.freq_grid_mbe(sets + [core_only], nfixed=10)
    assert np.array_equal(x1, x2)
    bad = (np.array([-1.0, 0.5, 0.2, 1.0]), 2, 2)  # HOMO above LUMO
    with pytest.raises(pkg.RPAError):
        pkg.freq_grid_mbe(sets + [bad], nfixed=10)


def test_pointer_classification_refuses_other_gpus(pkg, tmp_path):
    # the argument check of every entry point: device memory of another GPU is refused, the
    # handle's own device memory, managed memory and host memory pass (fake attribute values;
    # a single-GPU box cannot produce a real foreign pointer)
    import shutil
    import subprocess
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    src = tmp_path / "classify.cpp"
    src.write_text(r"""
#include "abi_guard.h"
#include <cstdio>
int main() {
  using rpa::ArgMemory;
  using rpa::classify_arg_memory;
  int bad = 0;
  // type: 0 unregistered host, 1 registered host, 2 device, 3 managed
  bad += classify_arg_memory(0, -2, 0) != ArgMemory::Host;
  bad += classify_arg_memory(1, 0, 1) != ArgMemory::Host;
  bad += classify_arg_memory(2, 0, 0) != ArgMemory::HandleDevice;
  bad += classify_arg_memory(2, 3, 3) != ArgMemory::HandleDevice;
  bad += classify_arg_memory(2, 1, 0) != ArgMemory::OtherDevice;
  bad += classify_arg_memory(2, 0, 7) != ArgMemory::OtherDevice;
  bad += classify_arg_memory(3, 5, 0) != ArgMemory::HandleDevice;
  std::printf("%d\n", bad);
  return bad;
}
""")
    exe = tmp_path / "classify"
    csrc = pkg.HEADER.parents[1] / "beyond-rpa_b200" / "csrc"
    subprocess.run([cxx, "-std=c++17", "-Wall", "-Werror", f"-I{csrc}", str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=30)
    assert out.returncode == 0 and out.stdout.strip() == "0", out.stdout


def test_every_entry_point_with_arrays_checks_their_device(pkg):
    # each entry point that takes array arguments runs check_arrays right after begin_call
    import re
    src = (pkg.HEADER.parents[1] / "beyond-rpa_b200" / "csrc" / "capi.cu").read_text()
    header = re.sub(r"/\*.*?\*/", " ", pkg.HEADER.read_text(), flags=re.S)
    with_arrays = [m.group(1) for m in re.finditer(r"^\s*int\s+(rpa_b200_\w+)\s*\(([^;]*?)\)\s*;", header, re.M)
                   if re.search(r"double\s*\*|rpa_instance\s*\*", m.group(2))]
    assert "rpa_b200_ec" in with_arrays
    for name in with_arrays:
        if name in ("rpa_b200_tune_logdet", "rpa_b200_freq_grid", "rpa_b200_freq_grid_mbe", "rpa_b200_mbe_energy",
                    "rpa_b200_last_timings", "rpa_b200_ec_from_pi_noalloc"):
            continue  # host-only arrays, or no handle (the no-alloc entry point has no handle device)
        body = src[src.index(f"\nint {name}("):]
        body = body[:body.index("\n} catch (...)")]
        assert "check_arrays(h, {" in body, name
