"""The C ABI library loads and exports every entry point include/tdfs.h
declares (no compute call: this runs without a GPU)."""
import os
import re
import subprocess

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def declared():
    text = open(os.path.join(ROOT, "include", "tdfs.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char \*)\s*(tdfs_\w+)\(", text, re.M)))


def test_header_and_exports_agree(T):
    names = declared()
    assert len(names) >= 20
    assert sorted(T.EXPORTS) == names
    lib = T.lib()
    for n in names:
        assert hasattr(lib, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", T.LIB_PATH], capture_output=True, text=True).stdout
    for n in names:
        assert re.search(rf"\bT {n}\b", out), n


def test_clis_built(T):
    for name in ("ulb", "lb"):
        assert os.access(os.path.join(T.BIN_DIR, name), os.X_OK)


def test_no_gpu_fails_loudly(T):
    import torch
    if torch.cuda.is_available():
        return
    g = T.gen_er(64, 4.0, 1)
    try:
        T.GraphPreprocessor(csr=g)
    except T.TdfsError as e:
        assert e.code == 4 and "no CUDA device" in str(e)
    else:
        raise AssertionError("graph upload must fail without a GPU")


def test_options_layout_matches_header(T, tmp_path):
    """The ctypes mirror of tdfs_options has the header's fields, in order, at
    the offsets a C compiler gives them (checked with gcc on the header)."""
    import ctypes
    import re
    import subprocess
    hdr = os.path.join(os.path.dirname(__file__), "..", "include", "tdfs.h")
    text = open(hdr).read()
    body = text[text.index("typedef struct {", text.index("Launch knobs")):text.index("} tdfs_options;")]
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    fields = re.findall(r"\b(\w+)\s*;", body)
    assert [f for f, _ in T.Options._fields_] == fields
    src = tmp_path / "layout.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "tdfs.h"\nint main(void) {\n'
                   '  printf("%zu\\n", sizeof(tdfs_options));\n' +
                   "".join(f'  printf("%zu\\n", offsetof(tdfs_options, {f}));\n' for f in fields) +
                   "  return 0;\n}\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.dirname(hdr), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert got[0] == ctypes.sizeof(T.Options)
    assert got[1:] == [getattr(T.Options, f).offset for f in fields]
