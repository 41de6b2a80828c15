"""The Fortran ISO_C_BINDING interfaces (fortran/imcom_gpu_iface.f90) against
the C declarations (include/imcom_gpu.h).

There is no Fortran compiler on either machine, so the interface module is
checked by parsing: every BIND(C, NAME=...) function must be declared in the
header with the same name, the same number of arguments and, argument by
argument, a matching C type -- a VALUE argument of INTEGER(C_INT),
INTEGER(C_LONG_LONG), REAL(C_DOUBLE) or TYPE(C_PTR) is passed by value (int,
long long, double, a pointer), every other argument by reference (a pointer
to the declared kind; a TYPE(C_PTR) without VALUE is a pointer to a pointer).
The checker itself is tested on mutated copies of the module (reordered
arguments, a dropped VALUE attribute, a changed kind), which it must reject.
"""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
F90 = os.path.join(ROOT, "fortran", "imcom_gpu_iface.f90")
HDR = os.path.join(ROOT, "include", "imcom_gpu.h")


def _join_continuations(text):
    out, buf = [], ""
    for raw in text.splitlines():
        line = raw.split("!", 1)[0].rstrip()
        if not line.strip():
            continue
        s = line.strip()
        if buf:
            s = s.lstrip("&").strip()
        if s.endswith("&"):
            buf += s[:-1] + " "
            continue
        out.append(buf + s)
        buf = ""
    return out


def parse_fortran(text):
    """{bind name: (return kind, [(kind, by_value) per argument in order])}."""
    lines = _join_continuations(text)
    body = []
    inside = False
    for ln in lines:
        up = ln.upper()
        if up.startswith("INTERFACE") and not inside:
            inside = True
            continue
        if up.startswith("END INTERFACE"):
            break
        if inside:
            body.append(ln)
    funcs, cur = {}, None
    head = re.compile(r"^(INTEGER\(C_INT\)|TYPE\(C_PTR\))\s+FUNCTION\s+(\w+)\s*\(([^)]*)\)\s*"
                      r"BIND\(C,\s*NAME=\"(\w+)\"\)", re.I)
    for ln in body:
        m = head.match(ln)
        if m:
            args = [a.strip().lower() for a in m.group(3).split(",") if a.strip()]
            cur = {"ret": "int" if m.group(1).upper().startswith("INTEGER") else "ptr",
                   "args": args, "decl": {}, "bind": m.group(4), "fname": m.group(2).lower()}
            funcs[cur["bind"]] = cur
            continue
        if ln.upper().startswith("END FUNCTION"):
            cur = None
            continue
        if cur is None or ln.upper().startswith("IMPORT"):
            continue
        if "::" not in ln:
            continue
        spec, names = ln.split("::", 1)
        su = spec.upper().replace(" ", "")
        kind = None
        for key, k in (("INTEGER(C_INT)", "int"), ("INTEGER(C_LONG_LONG)", "long long"),
                       ("REAL(C_DOUBLE)", "double"), ("REAL(C_FLOAT)", "float"),
                       ("TYPE(C_PTR)", "ptr"), ("CHARACTER(KIND=C_CHAR)", "char")):
            if su.startswith(key):
                kind = k
        assert kind is not None, f"unknown declaration: {ln}"
        value = ",VALUE" in su
        # names may carry their own dimensions, e.g. "A, Q" after DIMENSION(...)
        for nm in re.split(r",(?![^(]*\))", names):
            nm = nm.strip().split("(")[0].strip().lower()
            if nm:
                cur["decl"][nm] = (kind, value)
    out = {}
    for bind, f in funcs.items():
        missing = [a for a in f["args"] if a not in f["decl"]]
        assert not missing, f"{bind}: undeclared arguments {missing}"
        out[bind] = (f["ret"], [f["decl"][a] for a in f["args"]])
    return out


def parse_header(text):
    """{name: (return kind, [C type string per argument])}."""
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    text = re.sub(r"//[^\n]*", " ", text)
    out = {}
    for m in re.finditer(r"(int|const\s+char\s*\*)\s+(imcom_\w+)\s*\(([^;{]*?)\)\s*;", text):
        ret = "int" if m.group(1) == "int" else "ptr"
        args = [a.strip() for a in m.group(3).replace("\n", " ").split(",")]
        if args == ["void"]:
            args = []
        out[m.group(2)] = (ret, args)
    return out


def c_kind(arg):
    """(kind, pointer depth) of one C parameter declaration."""
    a = re.sub(r"\bconst\b", " ", arg)
    depth = a.count("*")
    a = a.replace("*", " ")
    toks = a.split()
    base = " ".join(toks[:-1]) if len(toks) > 1 else toks[0]
    return base, depth


def mismatches(fortran, header):
    bad = []
    for name, (fret, fargs) in fortran.items():
        if name not in header:
            bad.append(f"{name}: not declared in the header")
            continue
        hret, hargs = header[name]
        if fret != hret:
            bad.append(f"{name}: return kind {fret} vs {hret}")
        if len(fargs) != len(hargs):
            bad.append(f"{name}: {len(fargs)} arguments vs {len(hargs)}")
            continue
        for i, ((kind, value), carg) in enumerate(zip(fargs, hargs)):
            base, depth = c_kind(carg)
            if kind == "ptr":
                ok = depth == (1 if value else 2)
            elif value:
                ok = depth == 0 and base == kind
            else:
                ok = depth == 1 and base == kind
            if not ok:
                bad.append(f"{name}: argument {i + 1} is {kind}{' VALUE' if value else ''} in "
                           f"Fortran but '{carg}' in C")
    return bad


@pytest.fixture(scope="module")
def sources():
    return open(F90).read(), open(HDR).read()


def test_every_fortran_interface_matches_the_header(sources):
    f90, hdr = sources
    fortran, header = parse_fortran(f90), parse_header(hdr)
    assert len(fortran) >= 30, sorted(fortran)
    assert mismatches(fortran, header) == []


def test_header_functions_the_driver_calls_are_bound(sources):
    """Every entry point of the solve path's build branches has a Fortran binding."""
    f90, hdr = sources
    fortran = parse_fortran(f90)
    for name in ("imcom_gpu_create", "imcom_gpu_destroy", "imcom_gpu_set_inputs",
                 "imcom_gpu_set_psfs", "imcom_gpu_psf_spectra", "imcom_gpu_build_A",
                 "imcom_gpu_eigen_A", "imcom_gpu_build_B", "imcom_gpu_build_P",
                 "imcom_gpu_bisect_kappa", "imcom_gpu_build_T", "imcom_gpu_build_image",
                 "imcom_gpu_build_S", "imcom_gpu_build_U", "imcom_gpu_load_A",
                 "imcom_gpu_load_QL", "imcom_gpu_load_B", "imcom_gpu_load_P",
                 "imcom_gpu_load_T", "imcom_gpu_last_error", "imcom_fits_read",
                 "imcom_fits_write"):
        assert name in fortran, name


def _mutate(f90, func, old, new):
    i = f90.index(f'NAME="{func}"')
    j = f90.index("END FUNCTION", i)
    start = f90.rindex("FUNCTION", 0, i)
    start = f90.rindex("\n", 0, start)
    block = f90[start:j]
    assert old in block, (func, old)
    return f90[:start] + block.replace(old, new, 1) + f90[j:]


@pytest.mark.parametrize("func,old,new", [
    # two arguments of different kinds swapped in the argument list
    ("imcom_gpu_set_option", "(ctx, option, value)", "(ctx, value, option)"),
    ("imcom_gpu_build_U", "(ctx, C_a, U_out)", "(ctx, U_out, C_a)"),
    # a scalar passed by reference instead of by value
    ("imcom_gpu_build_A", "INTEGER(C_INT), VALUE :: npoly, npad", "INTEGER(C_INT) :: npoly, npad"),
    # a changed kind
    ("imcom_gpu_set_option", "INTEGER(C_LONG_LONG), VALUE :: value",
     "INTEGER(C_INT), VALUE :: value"),
    # an argument dropped
    ("imcom_gpu_load_QL", "(ctx, Q, L)", "(ctx, Q)"),
])
def test_checker_rejects_a_broken_interface(sources, func, old, new):
    f90, hdr = sources
    header = parse_header(hdr)
    bad_text = _mutate(f90, func, old, new)
    if new == "(ctx, Q)":
        bad_text = bad_text.replace("DIMENSION(*), INTENT(IN) :: Q, L", "DIMENSION(*), INTENT(IN) :: Q")
    bad = mismatches(parse_fortran(bad_text), header)
    assert any(b.startswith(func + ":") for b in bad), bad
