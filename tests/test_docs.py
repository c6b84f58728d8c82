"""The code in INTEGRATION.md stays valid: the ctypes stub a maintainer would add runs as written
against the built library (without a device its calls report errors through nmlmc_last_error
instead of exiting, so its final check becomes a print), and the C snippets of the native API
compile and link."""
import os
import re
import subprocess
import sys

from conftest import ROOT


def test_integration_ctypes_stub_runs():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    code = re.findall(r"```python\n(.*?)```", text, re.S)[0]
    assert "ctypes.CDLL" in code and "model_sample" in code
    code = code.replace("assert lib.nmlmc_last_error() == 0", "print('status', lib.nmlmc_last_error())")
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr[-2000:]
    assert "status" in out.stdout


def test_integration_c_snippets_compile_and_link(nm, tmp_path):
    """The C snippets of INTEGRATION.md compile as C99 against include/nmlmc.h and link against
    the library (not run: they need a device)."""
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    b0, b1, b2 = re.findall(r"```c\n(.*?)```", text, re.S)[:3]
    src = ("#include <stdint.h>\n#include <stddef.h>\n#include \"nmlmc.h\"\nint main(void) {\n" + b0 +
           "uint32_t ell = 3;\n" + b1 +
           "{\nconst uint32_t so[3] = {0, 1, 2}, oo[3] = {0, 1, 2}, si[2] = {0, 0};\n"
           "const int32_t ty[2] = {1, -1};\n"
           "const double S0[2] = {100, 90}, mu[2] = {0.05, 0.05}, sg[2] = {0.2, 0.3}, K[2] = {100, 95},"
           " T[2] = {1, 2}, w[2] = {1, -1}, Kloss[2] = {0, 0};\n"
           "double dEL_dw[2], dP_dw[2], dEL_dsigma[2], dP_dsigma[2];\n" + b2 + "}\n"
           "nmlmc_destroy(ctx);\nreturn 0;\n}\n")
    c = tmp_path / "snippets.c"
    c.write_text(src)
    libdir = os.path.dirname(nm.LIB_PATH)
    out = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-Wno-unused-variable",
                          f"-I{os.path.join(ROOT, 'include')}", str(c), "-o", str(tmp_path / "snippets"),
                          f"-L{libdir}", "-lnmlmc"], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr[-3000:]


def test_integration_cpp_snippet_compiles(nm, tmp_path):
    """The C++ snippet of INTEGRATION.md compiles as C++14 against include/nmlmc.hpp and links."""
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    code = re.findall(r"```cpp\n(.*?)```", text, re.S)[0]
    include, body = code.split("\n", 1)
    assert include.startswith("#include")
    src = ("#include <iostream>\n" + include + "\nint main() {\n"
           "uint32_t ell = 2; uint64_t M = 10, inner_stats[6]; double fsums[4], diffsums[4], work;\n"
           + body + "return 0;\n}\n")
    c = tmp_path / "snippet.cpp"
    c.write_text(src)
    libdir = os.path.dirname(nm.LIB_PATH)
    out = subprocess.run(["g++", "-std=c++14", "-Wall", "-Werror", "-Wno-unused-variable",
                          "-Wno-unused-parameter", f"-I{os.path.join(ROOT, 'include')}", str(c), "-o",
                          str(tmp_path / "snippet"), f"-L{libdir}", "-lnmlmc"], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr[-3000:]


def test_integration_python_snippets_parse():
    """Every Python snippet of INTEGRATION.md is valid Python (the multi-GPU one needs torchrun
    and GPUs to run)."""
    import ast
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    blocks = re.findall(r"```python\n(.*?)```", text, re.S)
    assert len(blocks) >= 2
    for b in blocks:
        ast.parse(b)


def test_docs_cite_files_that_exist():
    """Every repository file named in the user documentation (README.md: tests,
    profiles, sources, headers) exists; names of the reference's own files are not checked."""
    reference_files = {"common.cpp", "common.hpp", "mlmc.hpp", "model_sampler.cpp", "nested_sampler.hpp",
                       "par_nvcc.hpp", "par_omp.hpp", "portfolio_sampler.cpp", "gbm_approx.hpp",
                       "table_output.hpp", "threefry.h", "boxmuller.hpp", "uniform.hpp", "array.h",
                       "mlmc_test.cpp", "parse_mlmc_output.py", "my_main.cpp"}
    pkg = os.path.join(ROOT, "nested-risk-mlmc_b200")
    roots = [ROOT, pkg, os.path.join(pkg, "csrc"), os.path.join(pkg, "nmlmc"), os.path.join(ROOT, "oracle"),
             os.path.join(ROOT, "tests"), os.path.join(ROOT, "tests", "abi"), os.path.join(ROOT, "include")]
    missing = []
    for doc in ("INTEGRATION.md", "README.md"):
        text = open(os.path.join(ROOT, doc)).read()
        for m in re.finditer(r"[\w./-]+\.(?:py|md|cu|cuh|cpp|c|h|hpp|inc|json)\b", text):
            name = m.group(0).strip("./")
            if os.path.basename(name) in reference_files or name.startswith("_body"):
                continue
            if not any(os.path.exists(os.path.join(r, name)) for r in roots):
                missing.append((doc, name))
    assert not missing, missing
