"""The reference's own C ABI (libzebsdsolve.so, include/zebsdsolve.h) against the reference's binding
of it (python/zebsdsolve/_native.py:95-174, recorded in tests/golden/ze_abi.json by
tests/golden/make_ze_abi.py), on the CPU: every call the reference binds is exported and declared
with its argument and result kinds and sizes; the structs have its layouts, field for field, in the
header and in the package's ctypes mirror; the calls that need no GPU answer as the reference's do
(ze_version, a failed ze_create and its message, the engine's own frame, no WGSL)."""
import ctypes
import json
import re
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
GOLD = json.loads((ROOT / "tests" / "golden" / "ze_abi.json").read_text())
HEADER = ROOT / "include" / "zebsdsolve.h"

C_KINDS = {"void": ["none", 0], "uint32_t": ["uint", 4], "int32_t": ["int", 4], "uint64_t": ["uint", 8],
           "int64_t": ["int", 8], "size_t": ["uint", 8], "double": ["float", 8], "float": ["float", 4]}


def _lib_path():
    from zebsdsolve_b200 import build

    if not build.ABI_LIB.exists():
        build.build_abi()
    return build.ABI_LIB


def _c_kind(t):
    t = t.strip()
    if "*" in t:
        return ["ptr", 8]
    t = re.sub(r"\bconst\b", "", t).strip()
    return C_KINDS[t]


def _declarations():
    """name → (argument kinds, result kind) from the header's prototypes."""
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    out = {}
    for m in re.finditer(r"^([A-Za-z_][\w \t]*?[\s*]+)(ze_\w+)\s*\(([^;]*?)\)\s*;", text, flags=re.M):
        ret, name, args = m.group(1), m.group(2), " ".join(m.group(3).split())
        kinds = [] if args in ("", "void") else [_c_kind(re.sub(r"\s*\w+$", "", a.strip())) for a in args.split(",")]
        out[name] = (kinds, _c_kind(ret))
    return out


def test_every_reference_call_is_declared_with_its_kinds():
    decl = _declarations()
    missing = sorted(set(GOLD["sigs"]) - set(decl))
    assert not missing, missing
    for name, sig in GOLD["sigs"].items():
        args, ret = decl[name]
        assert args == sig["args"], (name, args, sig["args"])
        assert ret == sig["ret"], (name, ret, sig["ret"])


def test_the_library_exports_every_declared_call():
    """The 77 calls the reference's package binds and the 4 its web module adds (exports.zig)."""
    decl = _declarations()
    assert len(decl) == 81
    lib = ctypes.CDLL(str(_lib_path()))
    for name in decl:
        assert hasattr(lib, name), name


def test_structs_have_the_references_layouts():
    from zebsdsolve_b200 import ze_abi

    for name, s in GOLD["structs"].items():
        c = getattr(ze_abi, name)
        assert ctypes.sizeof(c) == s["size"], name
        ours = [(f, getattr(c, f).offset, getattr(c, f).size) for f, _ in c._fields_]
        assert [(o, z) for _, o, z in ours] == [(o, z) for _, o, z in s["fields"]], name


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_header_structs_have_the_references_layouts(tmp_path):
    lines = ["#include <stdio.h>", "#include <stddef.h>", f'#include "{HEADER}"', "int main(void) {"]
    for name, s in GOLD["structs"].items():
        lines.append(f'  printf("{name} %zu\\n", sizeof(ze_{name}));')
        for f, _, _ in s["fields"]:
            f = "pad" if f == "_pad" else f
            lines.append(f'  printf("{name}.{f} %zu\\n", offsetof(ze_{name}, {f}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", str(src), "-o", str(exe)], check=True)
    got = dict(line.rsplit(" ", 1) for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                               check=True).stdout.splitlines())
    for name, s in GOLD["structs"].items():
        assert int(got[name]) == s["size"], name
        for f, off, _ in s["fields"]:
            assert int(got[f"{name}.{'pad' if f == '_pad' else f}"]) == off, (name, f)


def test_calls_without_a_gpu():
    import torch

    lib = ctypes.CDLL(str(_lib_path()))
    lib.ze_version.restype = ctypes.c_char_p
    assert lib.ze_version() == b"0.2.8"
    buf = ctypes.create_string_buffer(512)
    lib.ze_frame.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]
    lib.ze_frame.restype = ctypes.c_size_t
    n = lib.ze_frame(None, buf, 512)
    assert json.loads(buf.raw[:n]) == {"axes": [1, 2, 3], "active": False, "crystal": "x_a_z_cstar",
                                       "text": "X +x Y +y Z +z, passive, X||a Z||c*"}
    lib.ze_shader.argtypes = [ctypes.c_uint32, ctypes.c_char_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t]
    lib.ze_shader.restype = ctypes.c_size_t
    assert lib.ze_shader(0, buf, 64, None, 0) == 0
    # a handle that is not an engine's: the call fails, nothing is touched
    lib.ze_configure.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]
    lib.ze_configure.restype = ctypes.c_int32
    assert lib.ze_configure(ctypes.c_void_p(0x10), b"{}", 2) < 0
    if not torch.cuda.is_available():
        lib.ze_create.argtypes = [ctypes.c_char_p]
        lib.ze_create.restype = ctypes.c_void_p
        assert not lib.ze_create(b"")
        lib.ze_create_error.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
        lib.ze_create_error.restype = ctypes.c_size_t
        n = lib.ze_create_error(buf, 512)
        assert b"no CUDA device" in buf.raw[:n]


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_a_native_host_starts_the_interpreter(tmp_path):
    """A C program (no Python process around it) linked against libzebsdsolve.so and libpython:
    the first call starts an interpreter, which finds the package beside the library; the calls
    answer as in a Python process (without a GPU, ze_create fails with ze_create_error's reason)."""
    import os
    import sys
    import sysconfig

    libdir, ldlib = sysconfig.get_config_var("LIBDIR"), sysconfig.get_config_var("LDLIBRARY")
    if not libdir or not ldlib or not os.path.exists(os.path.join(libdir, ldlib)):
        pytest.skip("no shared libpython to link")
    lib = _lib_path()
    src = tmp_path / "host.c"
    src.write_text("""#include <stdio.h>
#include "zebsdsolve.h"
int main(void) {
  char buf[512];
  void* e = ze_create("");
  size_t n = ze_create_error(buf, sizeof buf - 1);
  buf[n] = 0;
  printf("%s|%d|%s\\n", ze_version(), e != NULL, buf);
  if (e) ze_destroy(e);
  return 0;
}
""")
    exe = tmp_path / "host"
    py = ldlib[3:].split(".so")[0]  # libpython3.12.so -> python3.12
    subprocess.run(["gcc", str(src), "-I", str(HEADER.parent), "-L", str(lib.parent), "-lzebsdsolve", "-L", libdir,
                    f"-l{py}", f"-Wl,-rpath,{lib.parent}", f"-Wl,-rpath,{libdir}", "-o", str(exe)], check=True)
    env = dict(os.environ, PYTHONPATH=os.pathsep.join(p for p in sys.path if p))
    out = subprocess.run([str(exe)], capture_output=True, text=True, env=env, timeout=300)
    assert out.returncode == 0, out.stderr
    version, made, why = out.stdout.strip().splitlines()[-1].split("|", 2)
    import torch

    assert version == "0.2.8"
    if torch.cuda.is_available():
        assert made == "1"
    else:
        assert made == "0" and "no CUDA device" in why
