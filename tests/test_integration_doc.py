"""CPU: the examples of the integration guide compile against
include/asd2g.h (C, C++) or name the binding's real functions (Python), so
every documented call names a real entry point with the right arguments; the
repository paths the documents name exist."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# the names the examples leave to their surroundings; the batch examples use
# per-instance arrays for dt, iters and resid, the others scalars
COMMON = """
    asd2g_session *session = 0, *session2 = 0, *s = 0;
    asd2g_unet *net = 0;
    asd2g_batch *b = 0;
    asd2g_params params[4];
    void *stream = 0;
    int count = 4, nx = 64, ny = 64, it = 0, fell_back = 0, used = 0, i = 0, k = 0, K = 2;
    long long step = 0;
    double t = 0.0, first_dt = 1e-3, res = 0.0;
    const float *host_params = 0;
    const double *ls0 = 0;
    double *ls[2] = {0, 0}, *u[4] = {0}, *v[4] = {0}, *ps[2] = {0, 0}, *ps_i = 0;
"""
SCALARS = "    double dt = 1e-3, resid = 0.0; int iters = 0;\n"
ARRAYS = "    double dt[4] = {0}, resid[4] = {0}; int iters[4] = {0};\n"


def c_blocks():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    return re.findall(r"```c\n(.*?)```", text, re.S)


def test_integration_has_c_examples():
    assert len(c_blocks()) >= 4


@pytest.mark.parametrize("n", range(len(c_blocks())))
def test_c_example_compiles(tmp_path, n):
    block = c_blocks()[n]
    decls = COMMON + (ARRAYS if "asd2g_batch" in block else SCALARS)
    src = ('#include "asd2g.h"\nvoid example(void) {\n' + decls + "    {\n" + block + "\n    }\n}\n")
    path = tmp_path / f"example{n}.c"
    path.write_text(src)
    r = subprocess.run(["gcc", "-std=c11", "-fsyntax-only", "-Werror=implicit-function-declaration",
                        "-Werror=incompatible-pointer-types", "-Werror=int-conversion", "-Werror=return-type",
                        "-I", os.path.join(ROOT, "include"), str(path)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:] + "\n" + block


def cpp_blocks():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    return re.findall(r"```cpp\n(.*?)```", text, re.S)


@pytest.mark.parametrize("n", range(len(cpp_blocks())))
def test_cpp_example_compiles(tmp_path, n):
    """The C++ example, with its placeholder `...` for the first dt filled in
    and the caller's std::vector fields declared."""
    block = cpp_blocks()[n].replace("= ...;", "= 1e-3;")
    head = "\n".join(ln for ln in block.splitlines() if ln.startswith("#include"))
    body = "\n".join(ln for ln in block.splitlines() if not ln.startswith("#include"))
    src = (head + "\n#include <vector>\nvoid example() {\n    std::vector<double> ls, u, v, ps;\n" + body + "\n}\n")
    path = tmp_path / f"example{n}.cpp"
    path.write_text(src)
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I", os.path.join(ROOT, "include"), str(path)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:] + "\n" + block


def python_blocks():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    return re.findall(r"```python\n(.*?)```", text, re.S)


@pytest.mark.parametrize("n", range(len(python_blocks())))
def test_python_example_names_real_api(n):
    """The Python examples parse, and every api.* / workloads.* name and every
    Session method they call exists, with the keyword arguments they pass."""
    import ast
    import inspect

    from asd2_b200 import api
    from asd2_b200 import workloads as W
    tree = ast.parse(python_blocks()[n])
    modules = {"api": api, "W": W}
    for node in ast.walk(tree):
        if isinstance(node, ast.Attribute) and isinstance(node.value, ast.Name) and node.value.id in modules:
            assert hasattr(modules[node.value.id], node.attr), f"{node.value.id}.{node.attr}"
        if (isinstance(node, ast.Call) and isinstance(node.func, ast.Attribute)
                and isinstance(node.func.value, ast.Name) and node.func.value.id == "s"):
            meth = getattr(api.Session, node.func.attr, None)
            assert meth is not None, f"Session.{node.func.attr}"
            params = inspect.signature(meth).parameters
            for kw in node.keywords:
                assert kw.arg in params, f"Session.{node.func.attr}({kw.arg}=...)"


REPO_PREFIXES = ("asd2_b200/", "tests/", "oracle/", "include/", "profiles/")


@pytest.mark.parametrize("doc", ["DESIGN.md", "INTEGRATION.md", "README.md"])
def test_docs_name_existing_repo_files(doc):
    """Every repository path a document names in backticks exists (paths of
    the reference's own tree, such as src/mac2d.cpp, are not checked)."""
    text = open(os.path.join(ROOT, doc)).read()
    missing = []
    for m in re.finditer(r"`([A-Za-z0-9_./-]+)`", text):
        path = m.group(1).rstrip(".").split(":")[0]
        if path.startswith(REPO_PREFIXES) and "*" not in path and "_ref/" not in path:
            if not os.path.exists(os.path.join(ROOT, path)):
                missing.append(path)
    assert not missing, sorted(set(missing))
