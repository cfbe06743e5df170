"""The drop-in C ABI (include/ggems_api.h) against the reference's own
declarations: every extern "C" function of the reference's headers
(include/GGEMS/**, `extern "C" GGEMS_EXPORT ...`) outside the OpenGL
visualisation is declared here with the same name, the same number of
parameters and, parameter by parameter and for the return value, the same
calling-convention class (integer width and signedness, float / double, bool,
C string, opaque pointer); each declaration's citation names the reference
line that declares it.  Reads the reference checkout; skipped without it.
"""

import os
import re

import pytest

import parity

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
API = os.path.join(ROOT, "include", "ggems_api.h")

# type name -> calling-convention class
SCALARS = {
    "void": "void", "bool": "bool", "GGbool": "bool",
    "float": "f32", "GGfloat": "f32", "double": "f64", "GGdouble": "f64",
    "char": "i8", "GGchar": "i8", "int8_t": "i8", "GGuchar": "u8", "uint8_t": "u8", "unsigned char": "u8",
    "short": "i16", "GGshort": "i16", "int16_t": "i16", "GGushort": "u16", "uint16_t": "u16",
    "int": "i32", "GGint": "i32", "int32_t": "i32", "unsigned": "u32", "unsigned int": "u32", "GGuint": "u32",
    "uint32_t": "u32", "GGlong": "i64", "int64_t": "i64", "GGulong": "u64", "uint64_t": "u64", "GGsize": "u64",
    "size_t": "u64",
}
OPENGL = re.compile(r"opengl|_gl_|visualization", re.I)


def _class(decl):
    """Calling-convention class of a type written with or without a name."""
    decl = decl.split("=")[0].strip()                    # default argument
    decl = re.sub(r"\bconst\b", " ", decl)
    stars = decl.count("*")
    words = decl.replace("*", " ").split()
    base = " ".join(words)
    if base not in SCALARS and len(words) > 1:
        base = " ".join(words[:-1])                      # drop the parameter name
    if stars:
        return "cstr" if base in ("char", "GGchar") and stars == 1 else "ptr"
    if base not in SCALARS:
        raise AssertionError("unknown type %r" % decl)
    return SCALARS[base]


def _split(sig):
    m = re.match(r"\s*(.+?)\s*\b(\w+)\s*\((.*)\)\s*;", sig)
    assert m, sig
    ret, name, params = m.groups()
    params = [p for p in (x.strip() for x in params.split(",")) if p and p != "void"]
    return name, _class(ret), [_class(p) for p in params]


def _reference_declarations(ref):
    out = {}
    inc = os.path.join(ref, "include")
    for d, _, files in os.walk(inc):
        for f in files:
            path = os.path.join(d, f)
            for i, line in enumerate(open(path, errors="replace"), 1):
                if 'extern "C" GGEMS_EXPORT' in line:
                    sig = line.split('extern "C" GGEMS_EXPORT', 1)[1]
                    name, ret, params = _split(sig)
                    out[name] = (ret, params, os.path.relpath(path, ref), i)
    return out


def _our_declarations():
    out = {}
    for line in open(API):
        m = re.match(r"\s*([^/#{}]+?\));\s*/\*\s*(.*?)\s*\*/", line)
        if not m or "typedef" in line:
            continue
        name, ret, params = _split(m.group(1) + ";")
        out[name] = (ret, params, m.group(2))
    return out


@pytest.fixture(scope="module")
def reference():
    ref = parity.reference_dir()
    if ref is None:
        pytest.skip("reference checkout not available")
    return ref


def test_every_reference_function_is_declared_with_the_same_abi(reference):
    refs = _reference_declarations(reference)
    ours = _our_declarations()
    assert len(refs) > 150
    missing, wrong = [], []
    checked = 0
    for name, (ret, params, path, line) in sorted(refs.items()):
        if OPENGL.search(name):
            continue
        if name not in ours:
            missing.append(name)
            continue
        oret, oparams, cite = ours[name]
        if (oret, oparams) != (ret, params):
            wrong.append("%s: reference %s(%s), here %s(%s)" % (name, ret, ",".join(params), oret, ",".join(oparams)))
        assert cite == "%s:%d" % (path, line), (name, cite, path, line)
        checked += 1
    print("%d reference functions checked" % checked)
    assert not missing, missing
    assert not wrong, "\n".join(wrong)


def test_additions_are_marked(reference):
    """Functions with no reference counterpart say so in their citation."""
    refs = _reference_declarations(reference)
    for name, (_, _, cite) in _our_declarations().items():
        if name not in refs:
            assert "no counterpart in the reference" in cite, name
