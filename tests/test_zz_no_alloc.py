"""tbgpu_hx_dot_noalloc: H*x with the fused dot product, allocating nothing.

For callers that cannot let the library allocate (device memory handed to
their own pool allocator, or loops that cannot take cudaMalloc's device-wide
synchronisation), the library offers an H*x entry point whose reduction
scratch is a fixed array inside the library.  These tests call it through the
C ABI, twice in a row on the same buffers, and compare it with the regular
entry point tbgpu_hx_dev (same tolerance as the other H*x parity tests); the
dot product is compared with Re<x, y> of the regular result.  The file is
named to run last; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from nemo3d_b200 import materials, workloads

pytestmark = pytest.mark.gpu


def _lib():
    from nemo3d_b200 import tbgpu
    L = tbgpu._lib()
    L.tbgpu_hx_dot_noalloc.argtypes = [C.c_void_p, C.c_double, C.c_void_p, C.c_void_p,
                                       C.c_void_p]
    L.tbgpu_hx_dot_noalloc.restype = C.c_int
    return L


CASES = [
    ("sp3d5s*_so", ["GaAs_spds", "InAs_spds"],
     lambda: workloads.dome_in_box(cells=(9, 8, 7), base_nm=3.0, height_nm=1.2,
                                   wl_z_nm=1.4, sigma_frac=0.01, seed=4)),
    ("sp3d5s*", ["GaAs_spds", "InAs_spds"],
     lambda: workloads.dome_in_box(cells=(6, 7, 5), base_nm=2.0, height_nm=1.0,
                                   wl_z_nm=1.0, sigma_frac=0.01, seed=5)),
    ("sp3s*", ["GaAs_sps"], lambda: workloads.gaas_cube(6)),
]


@pytest.mark.parametrize("model,mats,make", CASES, ids=[c[0] for c in CASES])
def test_noalloc_matches_regular_entry_point(model, mats, make):
    import torch
    from nemo3d_b200.tbgpu import Hamiltonian
    torch.cuda.set_device(0)
    L = _lib()
    g = Hamiltonian(make(), model, [materials.MATERIALS[m] for m in mats])
    gen = torch.Generator(device="cuda").manual_seed(9)
    x = torch.rand(2 * g.n, dtype=torch.float64, device="cuda", generator=gen) - 0.5
    y_ref = torch.empty_like(x)
    shift = 0.35
    g.hx_dev(x.data_ptr(), y_ref.data_ptr(), shift)        # regular entry point
    torch.cuda.synchronize()
    dot_ref = torch.dot(x, y_ref).item()                    # Re<x, y>
    scale = y_ref.abs().max().item()
    for _ in range(2):                                      # two calls in a row
        y = torch.full_like(x, float("nan"))
        dot = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
        rc = L.tbgpu_hx_dot_noalloc(g._ctx, shift, x.data_ptr(), y.data_ptr(), dot.data_ptr())
        torch.cuda.synchronize()
        assert rc == 0
        assert (y - y_ref).abs().max().item() <= 1e-12 * scale
        assert abs(dot.item() - dot_ref) <= 1e-12 * abs(dot_ref) + 1e-12


def test_noalloc_refuses_launches_beyond_its_scratch():
    import torch
    from nemo3d_b200.tbgpu import Hamiltonian
    torch.cuda.set_device(0)
    L = _lib()
    g = Hamiltonian(workloads.gaas_cube(25), "sp3s*", [materials.MATERIALS["GaAs_sps"]])
    assert g.natoms > 98304
    x = torch.zeros(2 * g.n, dtype=torch.float64, device="cuda")
    y = torch.zeros_like(x)
    dot = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = L.tbgpu_hx_dot_noalloc(g._ctx, 0.0, x.data_ptr(), y.data_ptr(), dot.data_ptr())
    assert rc == -1   # TBGPU_E_ARG, refused on the host before any launch
