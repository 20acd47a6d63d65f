"""The Fortran binding module (include/mo_canard_gpu.f90) against the C header.

No Fortran compiler exists in this image, so the module is checked as text:
every entry point of include/canard_gpu.h has exactly one bind(C) interface
with the same name, the same number of arguments, and each argument passed
the way the C prototype takes it (by value for scalars and opaque handles,
by reference for arrays, out-arguments and strings); the drop-in module's
routines keep the reference's argument lists."""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
F90 = os.path.join(ROOT, "include", "mo_canard_gpu.f90")
HDR = os.path.join(ROOT, "include", "canard_gpu.h")


def c_prototypes():
    text = re.sub(r"/\*.*?\*/", "", open(HDR).read(), flags=re.S)
    out = {}
    for m in re.finditer(r"\n\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(canard_[a-z0-9_]+)\s*\(([^)]*)\)\s*;", text):
        params = [" ".join(p.split()) for p in m.group(2).split(",") if p.strip() and p.strip() != "void"]
        out[m.group(1)] = params
    return out


def by_value(cparam):
    """Scalars and opaque handles (canard_ctx*, void*) go by value."""
    stars = cparam.count("*")
    if stars == 0:
        return True
    base = re.sub(r"\bconst\b", "", cparam.split("*")[0]).strip()
    return stars == 1 and base in ("canard_ctx", "void")


def fortran_interfaces():
    src = open(F90).read()
    body = src.split("contains", 1)[0]  # the interface block of mo_canard_gpu
    src_lines = [ln.split("!")[0] for ln in body.splitlines()]
    text = "\n".join(src_lines).replace("&\n", " ")
    out = {}
    pat = re.compile(r"(?:integer\(\w+\)\s+function|type\(c_ptr\)\s+function|subroutine)\s+(\w+)\s*\(([^)]*)\)"
                     r"\s*bind\(C,\s*name=\"(\w+)\"\)(.*?)end\s+(?:function|subroutine)", re.S)
    for m in pat.finditer(text):
        args = [a.strip() for a in m.group(2).split(",") if a.strip()]
        decls = {}
        for line in m.group(4).splitlines():
            if "::" not in line:
                continue
            attrs, names = line.split("::", 1)
            a = attrs.replace(" ", "").lower()
            for nm in re.findall(r"(\w+)\s*(?:\([^)]*\))?", names):
                decls[nm] = ("value" in a.split(","), a.startswith("type(c_ptr)"))
        out[m.group(3)] = (m.group(1), args, decls)
    return out


def test_every_entry_point_has_one_interface():
    c = c_prototypes()
    f = fortran_interfaces()
    assert len(c) >= 40
    fnames = {k for k in f if k.startswith("canard_")}
    assert fnames == set(c), (sorted(set(c) - fnames), sorted(fnames - set(c)))
    assert "strlen" in f  # c_string's helper


@pytest.mark.parametrize("name", sorted(c_prototypes()))
def test_arguments_match_the_prototype(name):
    cparams = c_prototypes()[name]
    fname, args, decls = fortran_interfaces()[name]
    assert fname == name
    assert len(args) == len(cparams), (args, cparams)
    for a, p in zip(args, cparams):
        assert a in decls, f"{name}: {a} not declared"
        value, cptr = decls[a]
        if by_value(p):
            assert value, f"{name}: {a} ({p}) must be passed by value"
        else:
            # an array or out-argument by reference, or its address as type(c_ptr), value
            assert (not value) or cptr, f"{name}: {a} ({p}) must be passed by reference"


def test_helpers_and_dropin_routines_are_present():
    src = open(F90).read()
    assert re.search(r"function c_string\(p\)", src)
    assert re.search(r"subroutine canard_check\(rc, ctx, where\)", src)
    # the reference's argument lists (src/mo_physics.f90:216,306; src/mo_gcbc.f90:133,186,222;
    # src/mo_sponge.f90:75)
    for sig in (r"calc_viscous_shear_stress_gpu\(this, p_domdcomp, p_numerics, p_grid, de, ssk\)",
                r"calc_fluxes_gpu\(this, p_domdcomp, p_numerics, p_grid, qa, p, de\)",
                r"subroutine gcbc_setup\(p_domdcomp, p_numerics, p_grid, qa, p, de, umf\)",
                r"subroutine gcbc_comm\(p_domdcomp, p_numerics\)",
                r"subroutine gcbc_update\(p_domdcomp, p_numerics, p_grid, qa, p, de, nkrk, dt, umf, dudtmf\)",
                r"subroutine spongego\(lmx, qa, de\)"):
        assert re.search(sig, src), sig
    assert "procedure, public :: calc_fluxes => calc_fluxes_gpu" in src
    assert "procedure, public :: calc_viscous_shear_stress => calc_viscous_shear_stress_gpu" in src
