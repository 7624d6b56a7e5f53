"""The C ABI library loads and exports every symbol include/*.h declares.

No compute call is made here (no GPU on the CPU test host); only the host-only
entry points (version, file loaders, error reporting) are exercised.
"""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def _declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for dirpath, _, files in os.walk(inc):
        for f in files:
            if f.endswith(".h"):
                text = open(os.path.join(dirpath, f)).read()
                text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
                names |= set(re.findall(r"\b(ss_[a-z0-9_]+)\s*\(", text))
    return names


@pytest.fixture(scope="module")
def lib():
    from scattersearch_b200 import _native
    if not os.path.exists(_native.LIB_PATH):
        from scattersearch_b200 import build
        build.build()
    return _native.lib()


def test_every_declared_symbol_is_exported_and_bound(lib):
    from scattersearch_b200 import _native
    declared = _declared_symbols()
    assert len(declared) >= 20
    for name in sorted(declared):
        assert hasattr(lib, name), name
        assert name in _native.SIGNATURES, f"{name} has no ctypes signature"
    assert set(_native.SIGNATURES) <= declared


def test_version_and_error_reporting_without_gpu(lib):
    assert b"sm_100a" in lib.ss_version()
    h = ctypes.c_void_p()
    x = np.zeros((4, 8), np.float32)
    # bad arguments are rejected before any CUDA call
    rc = lib.ss_create(0, 4, x.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), 0, -1,
                       ctypes.byref(h))
    assert rc == 1 and b"nonzero" in lib.ss_last_error(None)
    rc = lib.ss_create(8, 4, x.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), 7, -1,
                       ctypes.byref(h))
    assert rc == 1 and b"metric" in lib.ss_last_error(None)


def test_host_loaders(lib, tmp_path):
    from scattersearch_b200 import io
    X = np.random.default_rng(0).standard_normal((7, 13)).astype(np.float32)
    p = str(tmp_path / "x.fbin")
    io.write_fbin(p, X)
    data = ctypes.POINTER(ctypes.c_float)()
    n, d = ctypes.c_uint32(), ctypes.c_uint32()
    assert lib.ss_load_fbin(p.encode(), ctypes.byref(data), ctypes.byref(n), ctypes.byref(d)) == 0
    got = np.ctypeslib.as_array(data, shape=(n.value * d.value + 8,)).copy()
    lib.ss_free(data)
    assert (n.value, d.value) == (7, 13)
    assert np.array_equal(got[:91].reshape(7, 13), X) and (got[91:] == 0).all()
    # truncated file is an error (the reference reads garbage)
    with open(p, "r+b") as f:
        f.truncate(8 + 4 * 50)
    assert lib.ss_load_fbin(p.encode(), ctypes.byref(data), ctypes.byref(n), ctypes.byref(d)) == 3
    assert lib.ss_load_fbin(b"/nonexistent/x.fbin", ctypes.byref(data), ctypes.byref(n),
                            ctypes.byref(d)) == 2
    gt = np.arange(12, dtype=np.uint32).reshape(3, 4)
    p = str(tmp_path / "gt.bin")
    io.write_groundtruth(p, gt)
    ids = ctypes.POINTER(ctypes.c_uint32)()
    nq, k = ctypes.c_uint32(), ctypes.c_uint32()
    assert lib.ss_load_groundtruth(p.encode(), ctypes.byref(ids), ctypes.byref(nq),
                                   ctypes.byref(k)) == 0
    got = np.ctypeslib.as_array(ids, shape=(12,)).copy()
    lib.ss_free(ids)
    assert (nq.value, k.value) == (3, 4) and np.array_equal(got.reshape(3, 4), gt)


def test_cpp_shim_compiles_against_the_abi(tmp_path):
    """The header-only ANNSearch shim builds with the system C++ compiler and
    links against the library (no run: that needs a GPU)."""
    import shutil
    import subprocess
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")
    if not cxx:
        pytest.skip("no C++ compiler")
    src = os.path.join(ROOT, "scattersearch_b200", "examples", "search_driver.cpp")
    out = str(tmp_path / "driver")
    lib_dir = os.path.join(ROOT, "scattersearch_b200")
    subprocess.run([cxx, "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), src, "-o", out,
                    "-L", lib_dir, "-lscattersearch_b200", "-Wl,-rpath," + lib_dir],
                   check=True)
    assert os.path.exists(out)


@pytest.mark.parametrize("driver", ["search", "parallel_search", "intraxinter",
                                    "online_parallel_search"])
def test_reference_drivers_compile_unchanged_against_the_dropin(tmp_path, driver):
    """The reference's benchmark drivers (its tests/*.cpp, read in place and
    not modified) compile and link against include/scattersearch/compat and
    the library: the compat headers supply everything the reference's
    include/annsearch.h and util.h supply (no run: that needs a GPU)."""
    import shutil
    import subprocess
    import __graft_entry__
    src = os.path.join(__graft_entry__.REFERENCE_SOURCES, "tests", f"{driver}.cpp")
    if not os.path.exists(src):
        pytest.skip("reference sources not present on this machine")
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")
    if not cxx:
        pytest.skip("no C++ compiler")
    out = str(tmp_path / driver)
    lib_dir = os.path.join(ROOT, "scattersearch_b200")
    subprocess.run([cxx, "-std=c++17", "-O2", "-fopenmp", "-pthread", "-I",
                    os.path.join(ROOT, "include", "scattersearch", "compat"), "-I",
                    os.path.join(ROOT, "include"), src, "-o", out, "-L", lib_dir,
                    "-lscattersearch_b200", "-Wl,-rpath," + lib_dir], check=True)
    assert os.path.exists(out)


def test_insert_into_pool_keeps_the_reference_contract(tmp_path):
    """compat/util.h's InsertIntoPool against the reference's (include/util.h:
    41-78, compiled from its header when present) on random pools with many
    exact distance ties and repeated ids."""
    import shutil
    import subprocess
    import __graft_entry__
    ref_inc = os.path.join(__graft_entry__.REFERENCE_SOURCES, "include")
    if not os.path.exists(os.path.join(ref_inc, "util.h")):
        pytest.skip("reference sources not present on this machine")
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")
    # one translation unit per implementation (same Neighbor layout), and a
    # driver comparing them on random pools
    wrap = r"""
#include <cstring>
#include <string>
#include <vector>
#include %s
extern "C" int %s(void *pool, unsigned K, unsigned id, float d) {
  return InsertIntoPool(static_cast<Neighbor *>(pool), K, Neighbor(id, d, true));
}
"""
    (tmp_path / "mine.cpp").write_text(wrap % ("<scattersearch/compat/util.h>", "mine_insert"))
    (tmp_path / "theirs.cpp").write_text(wrap % ("<util.h>", "theirs_insert"))
    (tmp_path / "main.cpp").write_text(r"""
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
struct N { unsigned id; float distance; bool unexplored; };
extern "C" int mine_insert(void *pool, unsigned K, unsigned id, float d);
extern "C" int theirs_insert(void *pool, unsigned K, unsigned id, float d);
int main() {
  srand(7);
  for (int t = 0; t < 200000; ++t) {
    unsigned K = 1 + rand() % 12;
    std::vector<N> a(K + 1), b(K + 1);
    float d = 0;
    for (unsigned i = 0; i < K; ++i) {
      d += (float)(rand() % 3);
      a[i] = b[i] = N{(unsigned)(rand() % 20), d, true};
    }
    float nd = (float)(rand() % (int)(d + 3)) - 1;
    unsigned nid = rand() % 20;
    int ra = mine_insert(a.data(), K, nid, nd);
    int rb = theirs_insert(b.data(), K, nid, nd);
    if (ra != rb) { printf("return %d vs %d at trial %d\n", ra, rb, t); return 1; }
    for (unsigned i = 0; i <= K; ++i)
      if (ra <= (int)K && (a[i].id != b[i].id || a[i].distance != b[i].distance)) {
        printf("slot %u differs at trial %d\n", i, t); return 1;
      }
  }
  printf("ok\n");
  return 0;
}
""")
    out = str(tmp_path / "pool")
    r2 = subprocess.run([cxx, "-std=c++17", "-O1", "-w", "-c", "-I", ref_inc,
                         str(tmp_path / "theirs.cpp"), "-o", str(tmp_path / "theirs.o")],
                        capture_output=True, text=True)
    assert r2.returncode == 0, r2.stderr[-3000:]
    r = subprocess.run([cxx, "-std=c++17", "-O1", "-w", "-I", os.path.join(ROOT, "include"),
                        str(tmp_path / "mine.cpp"), str(tmp_path / "main.cpp"),
                        str(tmp_path / "theirs.o"), "-o", out], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    run = subprocess.run([out], capture_output=True, text=True)
    assert run.returncode == 0 and "ok" in run.stdout, run.stdout
