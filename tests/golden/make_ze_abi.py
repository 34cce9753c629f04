"""Write tests/golden/ze_abi.json: the reference's C ABI as its Python package binds it
(python/zebsdsolve/_native.py:95-174 `_SIGS`, and its ctypes structs), for the tests that check
libzebsdsolve.so and include/zebsdsolve.h against it without the reference present.

    python tests/golden/make_ze_abi.py [<reference checkout>]

Each argument and result is recorded as its kind (ptr, int, uint, float, none) and size in bytes;
each struct as its fields' (name, offset, size) and its size.
"""
import ctypes
import importlib.util
import json
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent


def kind(t):
    if t is None:
        return ["none", 0]
    if t in (ctypes.c_char_p, ctypes.c_void_p) or hasattr(t, "_type_") and isinstance(t._type_, type):
        return ["ptr", ctypes.sizeof(ctypes.c_void_p)]
    if t in (ctypes.c_float, ctypes.c_double):
        return ["float", ctypes.sizeof(t)]
    return ["int" if t(-1).value < 0 else "uint", ctypes.sizeof(t)]


def main():
    ref = Path(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
    spec = importlib.util.spec_from_file_location("ref_native", ref / "python" / "zebsdsolve" / "_native.py")
    n = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(n)
    sigs = {name: {"args": [kind(a) for a in args], "ret": kind(res)} for name, (args, res) in n._SIGS.items()}
    structs = {}
    for name in ("ScanInfo", "PhaseInfo", "Geometry", "PcResult", "PlaneResult", "PlanePoint", "SimSummary",
                 "IndexStatus"):
        s = getattr(n, name)
        structs[name] = {"size": ctypes.sizeof(s),
                         "fields": [[f, getattr(s, f).offset, getattr(s, f).size] for f, _ in s._fields_]}
    out = {"source": "python/zebsdsolve/_native.py (zebsdsolve 0.2.8)", "sigs": sigs, "structs": structs}
    lines = ["{", f' "source": {json.dumps(out["source"])},', ' "sigs": {']
    lines += [f"  {json.dumps(k)}: {json.dumps(v)}," for k, v in sigs.items()]
    lines[-1] = lines[-1].rstrip(",")
    lines += [" },", ' "structs": {']
    lines += [f"  {json.dumps(k)}: {json.dumps(v)}," for k, v in structs.items()]
    lines[-1] = lines[-1].rstrip(",")
    lines += [" }", "}"]
    text = "\n".join(lines) + "\n"
    assert json.loads(text) == out
    (HERE / "ze_abi.json").write_text(text)
    print(f"{len(sigs)} calls, {len(structs)} structs")


if __name__ == "__main__":
    main()
