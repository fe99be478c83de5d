"""Import the reference's own ``ptychoX`` package from its install in ``baseline/_ref``.

``baseline/install_reference.sh`` installs the unmodified reference there; tests that need
it skip when the install is absent."""

import sys
from pathlib import Path

import pytest

REF_DIR = Path(__file__).resolve().parents[1] / "baseline" / "_ref"


def reference_package():
    if not (REF_DIR / "ptychoX" / "__init__.py").exists():
        pytest.skip("the reference is not installed in baseline/_ref (baseline/install_reference.sh)")
    if str(REF_DIR) not in sys.path:
        sys.path.insert(0, str(REF_DIR))
    import ptychoX

    assert Path(ptychoX.__file__).resolve().parent.parent == REF_DIR.resolve()
    return ptychoX
