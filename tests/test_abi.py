"""The C ABI: libnmlmc.so loads without a GPU, exports every function include/nmlmc.h declares,
and its structs have the reference's layout (sizes/offsets recorded from the reference build)."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT


def header_functions():
    src = open(os.path.join(ROOT, "include", "nmlmc.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = set()
    for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b([A-Za-z_]\w*)\s*\(([^;{]*?)\)\s*;", src, flags=re.M):
        if m.group(0).lstrip().startswith("typedef"):
            continue
        names.add(m.group(1))
    return names


def test_header_declares_all_exports(nm):
    declared = header_functions()
    assert declared == set(nm.EXPORTS), (declared ^ set(nm.EXPORTS))


def test_library_exports_every_declared_symbol(nm):
    lib = nm.lib()
    for name in header_functions():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", nm.LIB_PATH], capture_output=True, text=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l}
    assert header_functions() <= exported


def test_struct_layouts_match_reference(nm, golden):
    meta, _ = golden
    s = meta["abi_sizes"]
    assert ctypes.sizeof(nm.NestedSamplerParams) == s[0]
    assert ctypes.sizeof(nm.SampleOutput) == s[1]
    assert ctypes.sizeof(nm.ModelData) == s[2]
    assert ctypes.sizeof(nm.PortfolioData) == s[3]
    assert ctypes.sizeof(nm.OptionParams) == s[4]
    assert ctypes.sizeof(nm.StockParams) == s[5]
    assert nm.NestedSamplerParams.adaptive_r.offset == s[6]
    assert nm.SampleOutput.inner_stats.offset == s[7]
    assert nm.PortfolioData.subsample.offset == s[8]
    assert nm.PortfolioData.use_milstein.offset == s[9]
    assert nm.OptionParams.W_est.offset == s[10]
    assert nm.ModelData.phi_type.offset == s[11]


def test_error_strings_and_version(nm):
    lib = nm.lib()
    assert lib.nmlmc_version() >= 1
    for st in range(6):
        assert nm.error_string(st)


def test_no_device_is_an_error_not_a_fallback(nm):
    """Without a GPU the native API refuses (no CPU path exists)."""
    from conftest import HAVE_GPU
    if HAVE_GPU:
        pytest.skip("host has a GPU")
    with pytest.raises(nm.NmlmcError):
        nm.Sampler()


def test_plain_c_caller_builds_links_and_runs(nm, tmp_path):
    """The header is plain C (C99, -pedantic, no C++ or torch types): a C caller compiles, links
    against libnmlmc.so and calls the functions that need no device."""
    src = tmp_path / "caller.c"
    src.write_text(
        '#include <stdio.h>\n#include <string.h>\n#include "nmlmc.h"\n'
        "int main(void) {\n"
        "    nmlmc_mlmc_input in = nmlmc_mlmc_default_input();\n"
        "    if (nmlmc_version() <= 0) return 2;\n"
        "    if (strlen(nmlmc_error_string(NMLMC_ERR_ARG)) == 0) return 3;\n"
        "    printf(\"%d %g %u\\n\", nmlmc_version(), in.targetTOL, (unsigned)in.M0);\n"
        "    return 0;\n}\n")
    exe = tmp_path / "caller"
    libdir = os.path.dirname(nm.LIB_PATH)
    cc = subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror",
                         f"-I{os.path.join(ROOT, 'include')}", str(src), "-o", str(exe),
                         f"-L{libdir}", "-lnmlmc", f"-Wl,-rpath,{libdir}"],
                        capture_output=True, text=True)
    assert cc.returncode == 0, cc.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert run.returncode == 0, run.stderr
    v, tol, m0 = run.stdout.split()
    assert int(v) == nm.lib().nmlmc_version()


def test_null_arguments_are_errors_not_crashes(nm, tmp_path):
    """Each native entry point given a NULL context or NULL required pointers returns a status
    other than NMLMC_OK and does not crash (tests/abi/null_arguments.c)."""
    exe = tmp_path / "null_arguments"
    libdir = os.path.dirname(nm.LIB_PATH)
    cc = subprocess.run(["gcc", "-std=c99", "-Wall", f"-I{os.path.join(ROOT, 'include')}",
                         os.path.join(ROOT, "tests", "abi", "null_arguments.c"), "-o", str(exe),
                         f"-L{libdir}", "-lnmlmc", f"-Wl,-rpath,{libdir}"],
                        capture_output=True, text=True)
    assert cc.returncode == 0, cc.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120, cwd=tmp_path)
    assert run.returncode == 0, run.stdout + run.stderr
    assert "ok-calls 0" in run.stdout
    assert not (tmp_path / "x.ckpt").exists()


def test_reference_surface_out_of_order_is_recorded(nm, tmp_path):
    """The reference-named entry points, called before init or with NULL arguments, record an
    error (nmlmc_last_error) and return; the reference would exit() or crash there."""
    exe = tmp_path / "reference_surface_order"
    libdir = os.path.dirname(nm.LIB_PATH)
    cc = subprocess.run(["gcc", "-std=c99", "-Wall", f"-I{os.path.join(ROOT, 'include')}",
                         os.path.join(ROOT, "tests", "abi", "reference_surface_order.c"), "-o", str(exe),
                         f"-L{libdir}", "-lnmlmc", f"-Wl,-rpath,{libdir}"],
                        capture_output=True, text=True)
    assert cc.returncode == 0, cc.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120, cwd=tmp_path)
    assert run.returncode == 0, run.stdout + run.stderr
    assert "ok-calls 0" in run.stdout
    assert "failed" in run.stderr            # each error is also printed, as the reference prints


def test_cpp_entry_points(nm, tmp_path):
    """include/nmlmc.hpp: the driver's C++ interface (mlmc_real::run over a std::function level
    sampler) takes the C driver's decisions and prints its table, a sampler exception leaves run()
    unchanged, and sample<SAMPLER> before init is an error status (tests/abi/cpp_driver.cpp)."""
    exe = tmp_path / "cpp_driver"
    libdir = os.path.dirname(nm.LIB_PATH)
    cc = subprocess.run(["g++", "-std=c++14", "-Wall", "-Wextra", "-Werror",     # the reference's standard
                         f"-I{os.path.join(ROOT, 'include')}",
                         os.path.join(ROOT, "tests", "abi", "cpp_driver.cpp"), "-o", str(exe),
                         f"-L{libdir}", "-lnmlmc", f"-Wl,-rpath,{libdir}"],
                        capture_output=True, text=True)
    assert cc.returncode == 0, cc.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300, cwd=tmp_path)
    assert run.returncode == 0, run.stdout[-2000:] + run.stderr[-2000:]
    assert "ok-checks 0" in run.stdout


def test_norm_cdf_inv_export_matches_the_reference(nm, golden):
    """The exported norm_cdf_inv (host code; common.cpp:53-86 in real_t = float) returns the
    compiled reference's values bit for bit on the golden probabilities."""
    _, A = golden
    f = nm.lib().norm_cdf_inv
    f.restype = ctypes.c_float
    f.argtypes = [ctypes.c_float]
    got = np.array([f(float(p)) for p in A["ncdfinv/p"]], dtype=np.float32)
    np.testing.assert_array_equal(got.astype(np.float64), A["ncdfinv/f32"])


def test_python_constants_match_the_header(nm):
    """The binding's status, precision, stream-layout, model and sub-sampling constants have the
    values include/nmlmc.h gives them."""
    src = open(os.path.join(ROOT, "include", "nmlmc.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    values = {m.group(1): int(m.group(2)) for m in re.finditer(r"\b(NMLMC_[A-Z0-9_]+)\s*=\s*(-?\d+)", src)}
    pairs = {"NMLMC_OK": "OK", "NMLMC_ERR_ARG": "ERR_ARG", "NMLMC_ERR_CUDA": "ERR_CUDA",
             "NMLMC_ERR_STATE": "ERR_STATE", "NMLMC_ERR_NOMEM": "ERR_NOMEM",
             "NMLMC_ERR_TIMEOUT": "ERR_TIMEOUT", "NMLMC_ERR_LIMIT": "ERR_LIMIT",
             "NMLMC_PREC_REF32": "PREC_REF32", "NMLMC_PREC_FP64": "PREC_FP64", "NMLMC_PREC_FP32": "PREC_FP32",
             "NMLMC_STREAMS_CORE": "STREAMS_CORE", "NMLMC_STREAMS_OUTER": "STREAMS_OUTER",
             "NMLMC_MODEL_REFERENCE": "MODEL_REFERENCE", "NMLMC_MODEL_SHIFT": "MODEL_SHIFT",
             "NMLMC_SUB_NONE": "SUB_NONE", "NMLMC_SUB_RANDOM": "SUB_RANDOM", "NMLMC_SUB_UNIFORM": "SUB_UNIFORM"}
    for c_name, py_name in pairs.items():
        assert values[c_name] == getattr(nm, py_name), c_name


def test_ctypes_structs_match_the_c_header(nm, tmp_path):
    """Every struct of the Python binding has the size and field offsets the C compiler gives the
    header's struct of the same name (a mismatch would corrupt memory in the native calls)."""
    structs = {"NestedSamplerParams": "nested_sampler_params", "SampleOutput": "sample_output",
               "ModelData": "model_data", "OptionParams": "option_params", "StockParams": "stock_params",
               "PortfolioData": "portfolio_data", "Config": "nmlmc_config", "LevelResult": "nmlmc_level_result",
               "Portfolio": "nmlmc_portfolio", "PathMethods": "nmlmc_path_methods",
               "PortfolioBatch": "nmlmc_portfolio_batch", "AdjointConfig": "nmlmc_adjoint_config",
               "AdjointResult": "nmlmc_adjoint_result", "TraceRec": "nmlmc_trace_rec",
               "MlmcInput": "nmlmc_mlmc_input", "MlmcOutput": "nmlmc_mlmc_output",
               "PortfolioSpec": "nmlmc_portfolio_spec", "PhaseConfig": "nmlmc_phase_config",
               "CheckpointIO": "nmlmc_checkpoint_io"}
    lines, expect = [], {}
    for py, c in structs.items():
        cls = getattr(nm, py)
        lines.append(f'printf("{c} sizeof %zu\\n", sizeof({c}));')
        expect[(c, "sizeof")] = ctypes.sizeof(cls)
        for f in cls._fields_:
            lines.append(f'printf("{c} {f[0]} %zu\\n", offsetof({c}, {f[0]}));')
            expect[(c, f[0])] = getattr(cls, f[0]).offset
    src = tmp_path / "layout.c"
    src.write_text("#include <stddef.h>\n#include <stdio.h>\n#include \"nmlmc.h\"\nint main(void) {\n" +
                   "\n".join(lines) + "\nreturn 0;\n}\n")
    exe = tmp_path / "layout"
    cc = subprocess.run(["gcc", "-std=c99", f"-I{os.path.join(ROOT, 'include')}", str(src), "-o", str(exe)],
                        capture_output=True, text=True)
    assert cc.returncode == 0, cc.stderr[-3000:]
    got = {}
    for line in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines():
        c, field, value = line.split()
        got[(c, field)] = int(value)
    mismatched = {k: (expect[k], got[k]) for k in expect if expect[k] != got[k]}
    assert not mismatched, mismatched


def test_ctypes_argument_counts_match_the_header(nm):
    """Each function the binding declares argument types for takes as many arguments as its C
    prototype in include/nmlmc.h."""
    src = open(os.path.join(ROOT, "include", "nmlmc.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    protos = {}
    for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b([A-Za-z_]\w*)\s*\(([^;{]*?)\)\s*;", src, flags=re.M):
        if m.group(0).lstrip().startswith("typedef"):
            continue
        params = " ".join(m.group(2).split())
        protos[m.group(1)] = 0 if params in ("", "void") else params.count(",") + 1
    lib = nm.lib()
    checked = 0
    for name, n in protos.items():
        argtypes = getattr(lib, name).argtypes
        if argtypes is not None:
            assert len(argtypes) == n, (name, len(argtypes), n)
            checked += 1
    assert checked >= 20


def test_ctypes_result_types_match_the_header(nm):
    """Functions of the header that return something other than int or void have that result
    type in the binding (a float or struct read as int would be garbage)."""
    src = open(os.path.join(ROOT, "include", "nmlmc.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    want = {"uint64_t": ctypes.c_uint64, "const char*": ctypes.c_char_p, "float": ctypes.c_float,
            "portfolio_data": nm.PortfolioData, "nmlmc_mlmc_input": nm.MlmcInput}
    lib = nm.lib()
    seen = 0
    for m in re.finditer(r"^([A-Za-z_][\w \*]*?)\s*\b([A-Za-z_]\w*)\s*\(([^;{]*?)\)\s*;", src, flags=re.M):
        ret = " ".join(m.group(1).split()).replace(" *", "*")
        if ret.startswith("typedef") or ret in ("int", "void"):
            continue
        assert ret in want, (m.group(2), ret)
        assert getattr(lib, m.group(2)).restype == want[ret], m.group(2)
        seen += 1
    assert seen >= 5


@pytest.mark.parametrize("case", ["beta_overflow", "tau_nan", "max_loss_inf", "tau_above_one", "tau_below_zero"])
def test_noalloc_argument_checks(nm, case):
    """nmlmc_sample_level_noalloc rejects, before any device work, what nmlmc_set_model and
    nmlmc_sample reject: a level whose inner count N0 beta^ell overflows (beta = 65536, ell = 4:
    2^64 wraps to 0 as an integer power), non-finite tau or max_loss, and tau outside [0, 1] for
    the reference model; the status is also what nmlmc_last_error() reports afterwards."""
    lib = nm.lib()
    kind, tau, max_loss, beta, ell = nm.MODEL_SHIFT, 0.0, 1.0, 2, 3
    if case == "beta_overflow":
        beta, ell = 65536, 4
    elif case == "tau_nan":
        tau = float("nan")
    elif case == "max_loss_inf":
        max_loss = float("inf")
    elif case == "tau_above_one":
        kind, tau = nm.MODEL_REFERENCE, 1.5
    else:
        kind, tau = nm.MODEL_REFERENCE, -0.25
    # d_out is never dereferenced: every case is rejected before the device is touched
    rc = lib.nmlmc_sample_level_noalloc(kind, tau, max_loss, 32, beta, 1.5, 0, nm.PREC_FP32, 1, ell, 0, 1000,
                                        ctypes.c_void_p(256), None)
    assert rc == nm.ERR_ARG
    assert lib.nmlmc_last_error() == nm.ERR_ARG
