"""The Python binding refuses arrays whose shape, size, dtype or placement do not fit the block
before anything reaches the library: a wrong size would otherwise let a copy or a kernel read or
write past the caller's allocation.  Checked on the CPU with an engine object that has no
device context (every call below must stop in the binding)."""
import ctypes

import numpy as np
import pytest
import torch


@pytest.fixture()
def eng():
    from ocotillo_b200.engine import Engine, load_library
    e = Engine.__new__(Engine)
    e.lib, e.ctx, e.device, e.nw = load_library(), ctypes.c_void_p(), 0, 4
    return e


def test_host_solve_refuses_mismatched_arrays(eng):
    rho, T = np.ones((2, 3, 8)), np.ones((2, 3, 8))
    with pytest.raises(ValueError, match="one shape"):
        eng.solve_block(rho, np.ones((2, 3, 7)), 1e13)
    with pytest.raises(ValueError, match="one shape"):
        eng.solve_block(np.ones((6, 8)), np.ones((6, 8)), 1e13)
    with pytest.raises(ValueError, match="V: 5 elements where the block has 192"):
        eng.solve_block(rho, T, 1e13, out={"V": np.empty(5)})
    with pytest.raises(ValueError, match="contiguous float64"):
        eng.solve_block(rho, T, 1e13, out={"Vtop": np.empty((4, 2, 3), dtype=np.float32)})
    with pytest.raises(ValueError, match="contiguous float64"):
        eng.solve_block(rho, T, 1e13, out={"Vtop": np.empty((3, 2, 4)).T})


def test_device_solve_refuses_bad_tensors(eng):
    rho = torch.ones((2, 3, 8), dtype=torch.float64)
    with pytest.raises(ValueError, match="need a tensor on cuda:0"):  # right size, on the host
        eng.solve_block_device(rho, rho.clone(), 1e13, {})
    with pytest.raises(ValueError, match="rho: need a contiguous torch.float64"):
        eng.solve_block_device(rho.float(), rho, 1e13, {})
    with pytest.raises(ValueError, match="rho: need a contiguous torch.float64"):
        eng.solve_block_device(rho.transpose(0, 1), rho, 1e13, {})
    with pytest.raises(ValueError, match="shape"):
        eng.solve_block_device(rho.reshape(6, 8), rho.reshape(6, 8), 1e13, {})


def test_device_solve_checks_outputs_before_placement(eng, monkeypatch):
    """With inputs accepted, every named output must hold exactly its block's elements."""
    from ocotillo_b200 import engine as E
    seen = []

    def fake_need(name, t, numel, device, dtype=None):
        seen.append(name)
        if t.numel() != numel:
            raise ValueError(f"{name}: {t.numel()} elements where the block has {numel}")

    monkeypatch.setattr(E, "_need_tensor", fake_need)
    rho = torch.ones((2, 3, 8), dtype=torch.float64)
    with pytest.raises(ValueError, match="T: 47 elements where the block has 48"):
        eng.solve_block_device(rho, torch.ones(47, dtype=torch.float64), 1e13, {})
    with pytest.raises(ValueError, match="U: 10 elements where the block has 336"):
        eng.solve_block_device(rho, rho, 1e13, {"U": torch.empty(10)})
    with pytest.raises(ValueError, match="Vbot: 23 elements where the block has 24"):
        eng.solve_block_device(rho, rho, 1e13, {"Vtop": torch.empty(24), "Vbot": torch.empty(23)})
    with pytest.raises(ValueError, match="unknown array 'kapa'"):
        eng.solve_block_device(rho, rho, 1e13, {"kapa": torch.empty(192)})
    with pytest.raises(ValueError, match="Im: 191 elements"):
        eng.intensities_device(torch.empty(336), torch.empty(192), (2, 3, 8), 4, {"Ip": torch.empty(192),
                                                                                   "Im": torch.empty(191)})
    with pytest.raises(ValueError, match="kappa: 100 elements is not nw"):
        eng.optical_depth_device(torch.empty(100), rho, 1e13)
    with pytest.raises(ValueError, match="photo: 23 elements"):
        eng.optical_depth_device(torch.empty(192), rho, 1e13, photo=torch.empty(23))
    with pytest.raises(ValueError, match="V: 25 elements is not nw"):
        eng.integrated_flux_device(torch.empty(25), (2, 3))
    with pytest.raises(ValueError, match="out: 5 elements"):
        eng.integrated_flux_device(torch.empty(24), (2, 3), out=torch.empty(5))
    assert "U" in seen and "photo" in seen


def test_server_submit_refuses_mismatched_inputs():
    from ocotillo_b200 import Server
    s = Server.__new__(Server)
    with pytest.raises(ValueError, match="one shape"):
        s.submit(np.ones((2, 2, 8)), np.ones((2, 2, 9)), [5000.0], 1e13)
    with pytest.raises(ValueError, match="C-contiguous float64"):
        s.submit(np.ones((2, 2, 8), dtype=np.float32), np.ones((2, 2, 8)), [5000.0], 1e13)


def test_batch_bind_refuses_host_and_float32_tensors(eng):
    """The library bounds every column's range by the element counts it is given, which are
    only meaningful for float64 device arrays: anything else is refused in the binding."""
    from ocotillo_b200.engine import Batch
    b = Batch.__new__(Batch)
    b.eng, b.lib, b.offsets = eng, eng.lib, None
    x = torch.ones(64, dtype=torch.float64)
    with pytest.raises(ValueError, match="rho: need a tensor on cuda:0"):
        b.bind(x, x, {})
    with pytest.raises(ValueError, match="rho: need a contiguous torch.float64"):
        b.bind(x.float(), x, {})
    with pytest.raises(ValueError, match="unknown array 'Vtp'"):
        b.bind(x, x, {"Vtp": x})


def test_engine_close_closes_its_batches_first(eng):
    """A batch refers to its engine's context, so closing the engine closes its open batches
    before the context goes."""
    import weakref
    from ocotillo_b200.engine import Batch
    eng._batches = weakref.WeakSet()
    closed = []

    class FakeBatch(Batch):
        def close(self):
            closed.append(self)

    fb = FakeBatch.__new__(FakeBatch)
    eng._batches.add(fb)
    eng.close()
    assert closed == [fb]
