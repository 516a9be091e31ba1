"""The Julia drop-in files (julia/*.jl) against the C header.

Julia is not installed here, so the files cannot run; these checks read
them as text:
* every function of include/vsav.h has exactly one `ccall` binding in
  julia/libvsav.jl, with the argument and return types of its prototype;
* the Julia mirrors of the C structs have the C fields, in order, with
  matching types;
* both file sets (2D: Types/SpectralUtils/Utils/Init/Solvers/simulation,
  3D: the _3d twins) define the reference's API names, the step functions
  with the reference's argument counts (src/Solvers.jl:14,144,242,267,344,
  431,459), and blocks that open and close in balance.
"""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
JL = os.path.join(ROOT, "julia")
HEADER = os.path.join(ROOT, "include", "vsav.h")

SCALAR = {"int": "Cint", "int32_t": "Int32", "int64_t": "Int64", "uint64_t": "UInt64", "double": "Float64",
          "void": "Cvoid"}
POINTER = {"double": "Ptr{Float64}", "float": "Ptr{Float32}", "int32_t": "Ptr{Int32}", "int64_t": "Ptr{Int64}",
           "char": "Ptr{UInt8}", "void": "Ptr{Cvoid}", "vsav_handle": "Ptr{Cvoid}", "vsav_net": "Ptr{Cvoid}",
           "vsav_shape2d": "Ptr{VsavShape2D}", "vsav_config": "Ref{VsavConfig}",
           "vsav_options": "Ref{VsavOptions}", "vsav_status": "Ref{VsavStatus}"}
POINTER2 = {"vsav_handle": "Ptr{Ptr{Cvoid}}", "vsav_net": "Ptr{Ptr{Cvoid}}"}


def _strip_c_comments(s):
    return re.sub(r"/\*.*?\*/", "", s, flags=re.S)


def c_prototypes():
    s = _strip_c_comments(open(HEADER).read())
    out = {}
    for m in re.finditer(r"^\s*([\w\s\*]+?)\s*\b(vsav_\w+)\s*\(([^;{]*?)\)\s*;", s, flags=re.M):
        ret, name, args = m.group(1).strip(), m.group(2), " ".join(m.group(3).split())
        params = [] if args in ("", "void") else [a.strip() for a in args.split(",")]
        out[name] = (ret, params)
    return out


def julia_type_of(c_decl, is_return=False):
    """Julia ccall type of a C parameter declaration or return type."""
    d = c_decl.replace("const ", "").strip()
    stars = d.count("*")
    base = d.replace("*", " ").split()[0]
    if is_return and stars == 1 and base == "char":
        return "Cstring"
    if stars == 0:
        return SCALAR[base]
    if stars == 2:
        return POINTER2[base]
    return POINTER[base]


def julia_ccalls():
    s = open(os.path.join(JL, "libvsav.jl")).read()
    out = {}
    for m in re.finditer(r"ccall\(\(:(\w+),\s*libvsav\),\s*([\w{}]+),\s*\(([^()]*)\)", s):
        name, ret, args = m.group(1), m.group(2), m.group(3)
        types = [a.strip() for a in args.split(",") if a.strip()]
        assert name not in out, f"{name} bound twice"
        out[name] = (ret, types)
    return out


def test_every_header_function_is_bound_with_its_types():
    protos = c_prototypes()
    binds = julia_ccalls()
    assert len(protos) >= 45
    assert set(binds) == set(protos), (set(protos) ^ set(binds))
    for name, (ret, params) in protos.items():
        jret, jargs = binds[name]
        assert jret == julia_type_of(ret, is_return=True), (name, ret, jret)
        # a parameter is "type name": drop the name, keep the stars
        want = []
        for p in params:
            decl = re.sub(r"\b\w+$", "", p).strip() or p
            want.append(julia_type_of(decl))
        assert jargs == want, (name, params, jargs)


def c_struct_fields(cname):
    s = _strip_c_comments(open(HEADER).read())
    body = re.search(r"typedef struct %s \{(.*?)\}" % cname, s, flags=re.S).group(1)
    fields = []
    for decl in body.split(";"):
        decl = " ".join(decl.split())
        if not decl:
            continue
        m = re.match(r"(const )?([\w]+)(\s*\*?)\s*(.+)", decl)
        base, ptr, names = m.group(2), m.group(3).strip(), m.group(4)
        for nm in names.split(","):
            nm = nm.strip()
            arr = re.match(r"(\w+)\[(\d+)\]", nm)
            if ptr or nm.startswith("*"):
                fields.append((nm.lstrip("*"), "Ptr{%s}" % {"double": "Float64", "int32_t": "Int32"}[base]))
            elif arr:
                fields.append((arr.group(1), "NTuple{%s, %s}" % (arr.group(2), SCALAR[base])))
            else:
                fields.append((nm, SCALAR[base]))
    return fields


def julia_struct_fields(jname):
    s = open(os.path.join(JL, "libvsav.jl")).read()
    body = re.search(r"(?:mutable )?struct %s\n(.*?)\nend" % jname, s, flags=re.S).group(1)
    return [tuple(x.strip() for x in line.split("::")) for line in body.splitlines() if "::" in line]


@pytest.mark.parametrize("cname,jname", [("vsav_config", "VsavConfig"), ("vsav_options", "VsavOptions"),
                                         ("vsav_status", "VsavStatus"), ("vsav_shape2d", "VsavShape2D")])
def test_struct_mirrors_match_the_header(cname, jname):
    assert julia_struct_fields(jname) == c_struct_fields(cname)


def _code_only(s):
    """Julia source without comments and string literals (docstrings included)."""
    s = re.sub(r'"""(.*?)"""', '""', s, flags=re.S)
    s = re.sub(r'"(\\.|[^"\\])*"', '""', s)
    s = re.sub(r"#.*", "", s)
    return s


def block_balance(src):
    """Block openers minus `end`s outside () and [] (where `end` indexes and
    `for` / `if` build generators)."""
    s = _code_only(src)
    depth = 0
    bal = 0
    for tok in re.finditer(r"[()\[\]]|\b\w+\b", s):
        t = tok.group(0)
        if t in "([":
            depth += 1
        elif t in ")]":
            depth -= 1
        elif depth == 0:
            if t in ("function", "if", "for", "while", "begin", "let", "struct", "do", "try", "quote", "macro",
                     "module"):
                bal += 1
            elif t == "end":
                bal -= 1
    assert depth == 0
    return bal


def test_julia_blocks_balance():
    for f in sorted(os.listdir(JL)):
        if f.endswith(".jl"):
            assert block_balance(open(os.path.join(JL, f)).read()) == 0, f


def _defs(files):
    src = "\n".join(_code_only(open(os.path.join(JL, f)).read()) for f in files)
    defs = {}
    for m in re.finditer(r"(?:^|\n)\s*(?:function\s+)?([A-Za-z_][\w!]*)\s*\(([^()]*(?:\([^()]*\)[^()]*)*)\)\s*(?:=|\n|where)",
                         src):
        name, args = m.group(1), m.group(2)
        pos = args.split(";")[0]
        n = len([a for a in pos.split(",") if a.strip()])
        defs.setdefault(name, set()).add(n)
    structs = set(re.findall(r"struct\s+(\w+)", src))
    return defs, structs


SET_2D = ["Types.jl", "SpectralUtils.jl", "Utils.jl", "Init.jl", "Solvers.jl", "simulation.jl", "vsav_core.jl",
          "libvsav.jl"]
SET_3D = ["Types_3d.jl", "SpectralUtils_3d.jl", "Utils.jl", "Init_3d.jl", "Solvers.jl", "simulation.jl",
          "vsav_core.jl", "libvsav.jl"]
# argument counts of the reference's step functions (src/Solvers.jl:14,144,242,267,344,431,459)
STEP_ARGS = {"solve_step1": 6, "solve_step2": 6, "solve_step3": 2, "solve_step4": 5, "solve_step5": 7,
             "solve_step6": 4, "solve_step7": 5}


@pytest.mark.parametrize("files", [SET_2D, SET_3D], ids=["2d", "3d"])
def test_dropin_defines_the_reference_api(files):
    defs, structs = _defs(files)
    for s in ("Config", "FieldState", "Operators", "Step1Cache", "BDFCoeff"):
        assert s in structs, s
    for name, n in STEP_ARGS.items():
        assert n in defs.get(name, set()), (name, defs.get(name))
    assert 2 in defs["update_state!"]
    assert 1 in defs["build_operators"]
    for name in ("to_spectral!", "to_physical!"):
        assert 3 in defs[name], name
    assert 4 in defs["mult!"]
    assert 3 in defs["run_simulation"]
    assert 2 in defs["set_para_base"]
    assert 3 in defs["generate_initial_condition"]
    assert 3 in defs["calculate_area"]
    assert 4 in defs["compute_modified_energy"]
    assert {2, 3} & defs["download_state"]
    assert "upload_state!" in defs and "advance_state!" in defs
    assert "bdf_coeff" in defs


def test_the_3d_files_carry_3d_shapes():
    t = open(os.path.join(JL, "Types_3d.jl")).read()
    assert "phi::Array{Float64, 4}" in t and "Nz::Int" in t and "dz::Float64" in t
    s = open(os.path.join(JL, "SpectralUtils_3d.jl")).read()
    assert "ops.Nx * ops.Ny * ops.Nz" in s
