"""The C-ABI library loads and exports every entry point of include/dnsb.h.

No compute call is made here (no GPU needed).
"""

import re
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def _declared() -> set[str]:
    text = (ROOT / "include" / "dnsb.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(dnsb_\w+)\s*\(", text))


def test_library_exports_header():
    from dnsjax_b200 import _lib, build

    build.build()
    h = _lib.load()
    names = _declared()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(h, n)]
    assert not missing, missing
    # every declared entry point has a ctypes signature and vice versa
    assert names == set(_lib.SIGNATURES), names ^ set(_lib.SIGNATURES)
    assert h.dnsb_version() == 1


def test_product_does_not_import_oracle():
    pkg = ROOT / "dnsjax_b200"
    for f in pkg.rglob("*.py"):
        src = f.read_text()
        assert "import oracle" not in src and "from oracle" not in src, f
