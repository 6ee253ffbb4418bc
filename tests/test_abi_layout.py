"""The C ABI's struct layouts, three ways (CPU only):

- tests/abi_layout.c, compiled with gcc against include/pureadsorb_b200.h, prints sizeof and the
  offset of every field of every ABI struct;
- the ctypes mirrors in pureadsorb.jl_b200/_lib.py must have the same size, field names and offsets;
- the Julia structs of the binding in INTEGRATION.md must have the same fields in the same order,
  and their C layout (Julia `isbitstype` structs follow C alignment rules) the same offsets.
"""
import ctypes
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
C_OF_PY = {"pa_tuning": "Tuning", "pa_fp32_split": "Fp32Split", "pa_batch_desc": "BatchDesc",
           "pa_chain_args": "ChainArgs", "pa_widom_args": "WidomArgs", "pa_block_sums": "BlockSums",
           "pa_insertion_out": "InsertionOut", "pa_grad_sums": "GradSums"}
# the Julia structs the binding declares (the tuning struct is not used from Julia)
JULIA = {k: v for k, v in C_OF_PY.items() if k != "pa_tuning"}
JULIA_SIZE = {"Int32": 4, "UInt32": 4, "Int64": 8, "UInt64": 8, "Float64": 8, "Float32": 4}


@pytest.fixture(scope="module")
def c_layout(tmp_path_factory):
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("gcc not available")
    exe = str(tmp_path_factory.mktemp("abi") / "abi_layout")
    subprocess.run([gcc, "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "abi_layout.c"), "-o", exe], check=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    sizes, fields = {}, {}
    for line in out.splitlines():
        w = line.split()
        if w[0] == "struct":
            sizes[w[1]] = int(w[2])
            fields[w[1]] = []
        else:
            fields[w[1]].append((w[2], int(w[3])))
    return sizes, fields


def test_every_abi_struct_is_probed(c_layout):
    sizes, _ = c_layout
    with open(os.path.join(ROOT, "include", "pureadsorb_b200.h")) as fh:
        declared = set(re.findall(r"typedef struct (pa_\w+) \{", fh.read()))
    assert declared == set(sizes) == set(C_OF_PY)


def test_ctypes_mirrors_match_the_header(pa, c_layout):
    sizes, fields = c_layout
    for cname, pyname in C_OF_PY.items():
        st = getattr(pa._lib, pyname)
        assert ctypes.sizeof(st) == sizes[cname], cname
        assert [f[0] for f in st._fields_] == [f for f, _ in fields[cname]], cname
        for f, off in fields[cname]:
            assert getattr(st, f).offset == off, (cname, f)


def julia_structs():
    """{name: [(field, type)]} of every `struct` in the ```julia blocks of INTEGRATION.md."""
    with open(os.path.join(ROOT, "INTEGRATION.md")) as fh:
        text = fh.read()
    blocks = re.findall(r"```julia\n(.*?)```", text, re.S)
    out = {}
    for b in blocks:
        for name, body in re.findall(r"^struct (\w+)\n(.*?)^end", b, re.S | re.M):
            body = re.sub(r"#[^\n]*", "", body)
            out[name] = re.findall(r"(\w+)::([\w{}]+)", body)
    return out


def c_layout_of(fields):
    """(offsets, size) of a Julia isbits struct with these field types (C alignment rules)."""
    off, offs, align = 0, [], 1
    for _, t in fields:
        n = 8 if t.startswith("Ptr{") else JULIA_SIZE[t]
        off = (off + n - 1) // n * n
        offs.append(off)
        off += n
        align = max(align, n)
    return offs, (off + align - 1) // align * align


def test_julia_binding_structs_match_the_header(c_layout):
    sizes, fields = c_layout
    js = julia_structs()
    for cname, jname in JULIA.items():
        assert jname in js, jname
        jf = js[jname]
        assert [f for f, _ in jf] == [f for f, _ in fields[cname]], jname
        offs, size = c_layout_of(jf)
        assert offs == [o for _, o in fields[cname]], jname
        assert size == sizes[cname], jname
