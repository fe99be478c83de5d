"""The reference-side binding (``ptychox_b200.refshim``) on the host: it plugs into the
reference's own package and keeps the pybind11 extensions' argument checks (RuntimeError,
like TORCH_CHECK), without running a kernel."""

import pytest
import torch

from refpkg import reference_package


def test_install_sets_the_reference_extensions():
    ref = reference_package()
    from ptychox_b200 import refshim

    try:
        refshim.install(ref)
    except ImportError:
        pytest.skip("libptychox is not built")
    import ptychoX.base.ops as b
    import ptychoX.coded.ops as c
    import ptychoX.fpm.ops as f

    assert b._load_cuda_ext() is refshim.BASE
    assert f._load_cuda_ext() is refshim.FOURIER
    assert c._load_cuda_ext() is refshim.CODED
    b._CUDA_EXT = f._CUDA_EXT = c._CUDA_EXT = None


def test_extension_checks_raise_runtime_error():
    from ptychox_b200 import refshim

    s = torch.zeros(8, 8, dtype=torch.complex64)
    with pytest.raises(RuntimeError, match="sample must be a CUDA tensor"):
        refshim.BASE.forward(s, s, torch.zeros(1, 2, dtype=torch.long))
    with pytest.raises(RuntimeError, match="object_field must be a CUDA tensor"):
        refshim.FOURIER.forward(s, s, torch.zeros(1, 2, dtype=torch.long))
    with pytest.raises(RuntimeError, match="object must be a CUDA tensor"):
        refshim.CODED.forward(s, s, s, s, torch.zeros(1, 2), 2)
