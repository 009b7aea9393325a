"""The Zig binding (zig/src/backends/cuda_b200/ffi.zig) against the C ABI (include/stwo_b200.h).

No Zig toolchain is needed: both files are parsed as text. Every header function must have an
`extern fn` of the same name, arity and parameter types (integer widths, pointer depth and
constness, structs by value), and every header struct an `extern struct` (named by the typedef in
its doc comment) with the same fields in the same order; the structs' C layout (sizes and field
offsets, printed by a small C program built with gcc against the header) must equal the layout
of the Zig declarations under the C ABI rules that `extern struct` follows. Zig declarations
quoted in INTEGRATION.md are held to the same checks.
"""
import os
import re
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "stwo_b200.h")
FFI = os.path.join(ROOT, "zig", "src", "backends", "cuda_b200", "ffi.zig")
INTEGRATION = os.path.join(ROOT, "INTEGRATION.md")

C_BASE = {"uint8_t": "u8", "char": "u8", "uint32_t": "u32", "int32_t": "i32", "uint64_t": "u64",
          "size_t": "usize", "float": "f32", "double": "f64", "void": "void",
          "stwo_b200_context": "Context", "stwo_b200_server": "Server"}
ZIG_BASE = {"u8": "u8", "u32": "u32", "i32": "i32", "u64": "u64", "usize": "usize", "f32": "f32", "f64": "f64",
            "anyopaque": "void", "Context": "Context", "Server": "Server"}
SIZES = {"u8": 1, "u32": 4, "i32": 4, "u64": 8, "usize": 8, "f32": 4, "f64": 8}


def _strip_c(text):
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return re.sub(r"//[^\n]*", "", text)


def c_defines(text):
    return {m.group(1): int(m.group(2)) for m in re.finditer(r"#define\s+(\w+)\s+\(?(-?\d+)u?\)?", text)}


def c_type(decl, defines, param=False):
    """A C declarator ('const uint32_t* const* cols') -> (name, canonical type); an array
    parameter decays to a pointer."""
    toks = re.findall(r"\w+|\*|\[\w+\]", decl)
    arrays = [t for t in toks if t.startswith("[")]
    toks = [t for t in toks if not t.startswith("[")]
    name = toks[-1] if len(toks) > 1 and re.match(r"\w+$", toks[-1]) and toks[-1] not in C_BASE and \
        toks[-1] != "const" else None
    if name:
        toks = toks[:-1]
    base_const = False
    t = None
    i = 0
    while i < len(toks):
        tok = toks[i]
        if tok == "const":
            if t is None:
                base_const = True
            i += 1
            continue
        if tok == "*":
            pointee_const = base_const if isinstance(t, str) else t_const
            t = ("ptr", t, pointee_const)
            t_const = False
            if i + 1 < len(toks) and toks[i + 1] == "const":
                t_const = True
                i += 1
        else:
            t = C_BASE.get(tok, tok)
            t_const = base_const
        i += 1
    if param and arrays:
        return name, ("ptr", t, t_const)
    for dim in reversed(arrays):
        n = dim[1:-1]
        t = ("arr", int(defines.get(n, n)), t)
    return name, t


def parse_header(path=HEADER):
    raw = open(path).read()
    defines = c_defines(raw)
    text = _strip_c(raw)
    structs = {}
    for m in re.finditer(r"typedef\s+struct\s*\{(.*?)\}\s*(\w+)\s*;", text, flags=re.S):
        fields = []
        for stmt in m.group(1).split(";"):
            stmt = " ".join(stmt.split())
            if not stmt:
                continue
            parts = stmt.split(",")
            _, first_t = c_type(parts[0], defines)
            first_name, _ = c_type(parts[0], defines)
            base = re.match(r"((?:const\s+)?\w+)", parts[0]).group(1)
            fields.append((first_name, first_t))
            for extra in parts[1:]:
                fields.append(c_type(base + " " + extra, defines))
        structs[m.group(2)] = fields
    funcs = {}
    for m in re.finditer(r"((?:const\s+)?\w+\s*\**)\s*(stwo_b200_\w+)\s*\(([^)]*)\)\s*;", text):
        params = [] if m.group(3).strip() == "void" else [c_type(p, defines, True)[1] for p in m.group(3).split(",")]
        funcs[m.group(2)] = (c_type(m.group(1) + " x", defines)[1], params)
    return structs, funcs, defines


def zig_type(s, consts, names):
    s = s.strip()
    if s.startswith("?"):
        return zig_type(s[1:], consts, names)
    m = re.match(r"^(\*|\[\*(?::0)?\])\s*(const\s+)?(.*)$", s)
    if m:
        inner = zig_type(m.group(3), consts, names)
        if isinstance(inner, tuple) and inner[0] == "arr":  # a pointer to an array: the C array parameter
            return ("ptr", inner[2], bool(m.group(2)))
        return ("ptr", inner, bool(m.group(2)))
    m = re.match(r"^\[(\w+)\](.*)$", s)
    if m:
        n = m.group(1)
        return ("arr", int(consts.get(n, n)), zig_type(m.group(2), consts, names))
    return ZIG_BASE.get(s, names.get(s, s))


def parse_zig(text, known=""):
    """extern structs and fns of `text`; `known` is Zig source whose declarations `text` may use
    (struct names and constants)."""
    consts = {m.group(1): int(m.group(2))
              for m in re.finditer(r"pub const (\w+)(?::\s*\w+)?\s*=\s*(-?\d+);", known + text)}
    names = {}
    for m in re.finditer(r"((?:///[^\n]*\n)*)pub const (\w+) = extern struct", known):
        doc = re.search(r"(stwo_b200_\w+)", m.group(1))
        if doc:
            names[m.group(2)] = doc.group(1)
    structs = {}
    for m in re.finditer(r"((?:///[^\n]*\n)*)pub const (\w+) = extern struct \{(.*?)\n\};", text, flags=re.S):
        doc = re.search(r"(stwo_b200_\w+)", m.group(1))
        assert doc, f"extern struct {m.group(2)} has no doc comment naming its C typedef"
        names[m.group(2)] = doc.group(1)
    for m in re.finditer(r"pub const (\w+) = extern struct \{(.*?)\n\};", text, flags=re.S):
        fields = []
        for line in m.group(2).split("\n"):
            line = line.split("//")[0].strip().rstrip(",")
            if line:
                fname, ftype = line.split(":", 1)
                fields.append((fname.strip(), zig_type(ftype, consts, names)))
        structs[names[m.group(1)]] = fields
    funcs = {}
    for m in re.finditer(r"pub extern fn (\w+)\((.*?)\)\s*([^;]+);", text, flags=re.S):
        params = [p for p in (x.strip() for x in m.group(2).split(",")) if p]
        funcs[m.group(1)] = (zig_type(m.group(3), consts, names),
                             [zig_type(p.split(":", 1)[1], consts, names) for p in params])
    return structs, funcs


def layout(t, structs):
    """(size, align) of a canonical type under the C ABI (x86-64 / aarch64 LP64)."""
    if isinstance(t, tuple) and t[0] == "ptr":
        return 8, 8
    if isinstance(t, tuple) and t[0] == "arr":
        s, a = layout(t[2], structs)
        return s * t[1], a
    if t in SIZES:
        return SIZES[t], SIZES[t]
    off, al = 0, 1
    for _, ft in structs[t]:
        s, a = layout(ft, structs)
        off = (off + a - 1) // a * a + s
        al = max(al, a)
    return (off + al - 1) // al * al, al


def offsets(name, structs):
    out, off = [], 0
    for fname, ft in structs[name]:
        s, a = layout(ft, structs)
        off = (off + a - 1) // a * a
        out.append((fname, off))
        off += s
    return out


def c_layouts(structs):
    src = ['#include <stddef.h>', '#include <stdio.h>', f'#include "{HEADER}"', "int main(void) {"]
    for name, fields in structs.items():
        src.append(f'  printf("{name} %zu\\n", sizeof({name}));')
        for fname, _ in fields:
            src.append(f'  printf("{name}.{fname} %zu\\n", offsetof({name}, {fname}));')
    src.append("  return 0;\n}")
    with tempfile.TemporaryDirectory() as d:
        c, exe = os.path.join(d, "layout.c"), os.path.join(d, "layout")
        open(c, "w").write("\n".join(src))
        subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", c, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    return {k: int(v) for k, v in (line.split() for line in out.splitlines())}


@pytest.fixture(scope="module")
def header():
    return parse_header()


@pytest.fixture(scope="module")
def ffi():
    return parse_zig(open(FFI).read())


def test_every_header_function_is_declared_with_the_same_signature(header, ffi):
    _, cfuncs, _ = header
    _, zfuncs = ffi
    assert set(cfuncs) == set(zfuncs), (sorted(set(cfuncs) - set(zfuncs)), sorted(set(zfuncs) - set(cfuncs)))
    for name, (cret, cparams) in cfuncs.items():
        zret, zparams = zfuncs[name]
        assert zret == cret, (name, "return", zret, cret)
        assert len(zparams) == len(cparams), (name, "arity", len(zparams), len(cparams))
        for i, (z, c) in enumerate(zip(zparams, cparams)):
            assert z == c, (name, i, z, c)


def test_every_header_struct_is_declared_field_by_field(header, ffi):
    cstructs, _, _ = header
    zstructs, _ = ffi
    assert set(cstructs) == set(zstructs), (set(cstructs) ^ set(zstructs))
    for name, fields in cstructs.items():
        assert zstructs[name] == fields, (name, zstructs[name], fields)


def test_struct_layouts_match_the_c_compiler(header, ffi):
    cstructs, _, _ = header
    zstructs, _ = ffi
    measured = c_layouts(cstructs)
    for name in cstructs:
        assert layout(name, zstructs)[0] == measured[name], (name, layout(name, zstructs), measured[name])
        for fname, off in offsets(name, zstructs):
            assert off == measured[f"{name}.{fname}"], (name, fname, off)


def test_constants_match_the_header(header):
    _, _, defines = header
    text = open(FFI).read()
    for zname, cname in [("E_INVALID", "STWO_B200_E_INVALID"), ("E_OOM", "STWO_B200_E_OOM"),
                         ("E_TIMEOUT", "STWO_B200_E_TIMEOUT"), ("E_REJECTED", "STWO_B200_E_REJECTED"),
                         ("E_DIVISION_BY_ZERO", "STWO_B200_E_DIVISION_BY_ZERO"),
                         ("TRACE_FIRST_COLUMNS", "STWO_B200_TRACE_FIRST_COLUMNS"),
                         ("SERVER_VERIFY", "STWO_B200_SERVER_VERIFY"),
                         ("SERVER_PERSISTENT_WORKSPACES", "STWO_B200_SERVER_PERSISTENT_WORKSPACES"),
                         ("NOALLOC_EVAL_SCRATCH", "STWO_B200_NOALLOC_EVAL_SCRATCH"),
                         ("EVAL_AT_POINT_MAX_COLS", "STWO_B200_EVAL_AT_POINT_MAX_COLS"),
                         ("MAX_POW_BITS", "STWO_B200_MAX_POW_BITS"), ("LOGUP_MAX_WORDS", "STWO_B200_LOGUP_MAX_WORDS")]:
        m = re.search(rf"pub const {zname}(?::\s*\w+)?\s*=\s*(-?\d+);", text)
        assert m and int(m.group(1)) == defines[cname], zname


def test_integration_doc_points_at_the_binding_and_quotes_it_faithfully(header):
    doc = open(INTEGRATION).read()
    for path in ("zig/src/backends/cuda_b200/ffi.zig", "zig/src/backends/cuda_b200/commit_backend.zig",
                 "zig/build_support/backends/cuda_b200.zig"):
        assert path in doc and os.path.exists(os.path.join(ROOT, path)), path
    cstructs, cfuncs, _ = header
    zig_blocks = "\n".join(re.findall(r"```zig\n(.*?)```", doc, flags=re.S))
    zstructs, zfuncs = parse_zig(zig_blocks, known=open(FFI).read())
    for name, fields in zstructs.items():
        assert fields == cstructs[name], name
    for name, (ret, params) in zfuncs.items():
        assert (ret, params) == cfuncs[name], name


def test_the_parsers_see_what_they_check():
    # A declaration that drifts from the header is caught: a missing field and a narrowed width.
    structs, _, _ = parse_header()
    bad = parse_zig("/// stwo_b200_server_config\npub const ServerConfig = extern struct {\n"
                    "    slots: u32,\n    profile: u32,\n    memory_budget: u64,\n};\n")[0]
    assert bad["stwo_b200_server_config"] != structs["stwo_b200_server_config"]
    _, funcs, _ = parse_header()
    _, zf = parse_zig("pub extern fn stwo_b200_pow_grind(ctx: *Context, prefix_digest: *const [32]u8, "
                      "n_bits: u32, nonce_out: *u32) i32;")
    assert zf["stwo_b200_pow_grind"] != funcs["stwo_b200_pow_grind"]
    assert funcs["stwo_b200_merkle_commit_lifted"][1][2] == ("ptr", ("ptr", "u32", True), True)
