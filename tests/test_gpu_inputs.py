"""The synthetic disk inputs generated on the GPU (oco_disk_inputs_device) equal the host
generator's (oco_disk_inputs) bit for bit: the reference's disk model (disk.f90:42-129) with and
without the seeded lognormal perturbation, a ragged shape, and the precision and serving
constructions the benchmark generates in HBM."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape,kw", [((4, 5, 96), {}),
                                      ((3, 7, 257), {"sigma_dex": 0.3, "seed": 2}),
                                      ((16, 16, 1024), {"rho0": 3e-10, "sigma_dex": 0.3, "seed": 1003}),
                                      ((2, 3, 40), {"isoTemp": 1.0, "midTemp": 1.0, "sigma_dex": 0.5, "seed": 7}),
                                      ((1, 1, 2), {"rho_floor": 1e-15, "sigma_dex": 0.1, "seed": 2 ** 40 + 5})])
def test_device_inputs_equal_host(shape, kw):
    import torch
    from ocotillo_b200 import Engine, disk_inputs
    eng = Engine(0)
    dev = torch.device("cuda:0")
    rho = torch.full(shape, float("nan"), dtype=torch.float64, device=dev)
    T = torch.full(shape, float("nan"), dtype=torch.float64, device=dev)
    dz = eng.disk_inputs_device(rho, T, kw)
    torch.cuda.synchronize()
    rh, Th, dzh = disk_inputs(shape, **kw)
    assert dz == dzh
    assert np.array_equal(rho.cpu().numpy().view(np.uint64), rh.view(np.uint64))
    assert np.array_equal(T.cpu().numpy().view(np.uint64), Th.view(np.uint64))
    eng.close()


def test_serving_job_inputs_on_device():
    import torch
    from ocotillo_b200 import Engine, disk_inputs, workloads
    eng = Engine(0)
    job = workloads.serving_stream(3, 1.0, seed=5)[2]
    job = dict(job, nx=8, ny=8)
    rho, T, dz = workloads.job_arrays_device(job, eng)
    torch.cuda.synchronize()
    rh, Th, _ = disk_inputs((8, 8, job["nz"]), rho0=job["rho0"], sigma_dex=0.3, seed=job["seed"])
    assert np.array_equal(rho.cpu().numpy(), rh) and np.array_equal(T.cpu().numpy(), Th)
    eng.close()
