"""include/nf_capi.h is valid C11 and C++17 (the languages of a cgo / ctypes
binding and of abacus' own shim), declares every entry point as a function,
and its descriptor structs initialise the way the integration guide fills
them.  Compiled from standard input to /dev/null: nothing is written."""
import pathlib
import shutil
import subprocess

import pytest

INCLUDE = pathlib.Path(__file__).resolve().parents[1] / "include"


def _source(capi, lang):
    names = capi.declared_symbols()
    body = "\n".join(f"    (void)&{n};" for n in names)
    zero = "{}" if lang == "c++" else "{0}"
    return f"""#include "nf_capi.h"
int check_header(void);
int check_header(void) {{
{body}
    nf_sic_desc d = {zero};
    d.node_z_start = 3;
    d.node_z_size = 5;
    nf_driver_params p = {zero};
    p.node_z_start = d.node_z_start;
    p.node_z_size = d.node_z_size;
    return NF_ABI_VERSION + d.nk + p.cpd;
}}
"""


@pytest.mark.parametrize("lang,compiler,std", [("c", "gcc", "-std=c11"), ("c++", "g++", "-std=c++17")])
def test_header_compiles(capi, lang, compiler, std):
    if shutil.which(compiler) is None:
        pytest.skip(f"{compiler} not found")
    r = subprocess.run([compiler, "-pipe", "-x", lang, std, "-Wall", "-Wextra", "-Werror", "-pedantic",
                        f"-I{INCLUDE}", "-c", "-", "-o", "/dev/null"],
                       input=_source(capi, lang), capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_abi_version_matches_binding(capi):
    text = (INCLUDE / "nf_capi.h").read_text()
    assert f"#define NF_ABI_VERSION {capi.ABI_VERSION}" in text
