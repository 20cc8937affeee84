"""Athena snapshots from disk into HBM (oco_deck_block_inputs_device): the device reassembles
each processor block from its z-block files and applies the reader's physics
(read_athena.f90:101-277: momentum-underflow rule, T from E, unit system, density floor;
calc_temperature disk.f90:64-109) with the host reader's operations, so rho and T equal
oco_deck_block_inputs bit for bit; a deck block goes through the serving loop as a job."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("deck", ["ReadFromAthena", "multiInTest", "NongreyAGN"])
def test_device_block_inputs_equal_host(deck):
    from conftest import SAMPLES
    from ocotillo_b200 import Engine, deck_block_inputs
    path = os.path.join(SAMPLES, deck)
    eng = Engine(0)
    h0 = deck_block_inputs(path)
    for ipx in range(h0["nprocx"]):
        for ipy in range(h0["nprocy"]):
            h = deck_block_inputs(path, iprocx=ipx, iprocy=ipy)
            d = eng.deck_block_inputs_device(path, iprocx=ipx, iprocy=ipy)
            for k in ("rho", "T"):
                assert np.array_equal(d[k].cpu().numpy().view(np.uint64), h[k].view(np.uint64)), (deck, ipx, ipy, k)
            assert np.array_equal(d["z"], h["z"]) and np.array_equal(d["wa"], h["wa"]) and d["dz"] == h["dz"]
    eng.close()


def test_athena_deck_as_a_serving_job():
    from conftest import SAMPLES
    from ocotillo_b200 import Engine, Server, deck_block_inputs
    path = os.path.join(SAMPLES, "multiInTest")
    eng = Engine(0)
    srv = Server(0, max_jobs=2, max_nz=64)
    jid, info = srv.submit_deck(eng, path, iprocx=1, iprocy=0, form="plain")
    srv.wait(jid, 120.0)
    got = srv.fetch(jid)
    srv.close()
    h = deck_block_inputs(path, iprocx=1, iprocy=0)
    eng.set_wavelengths(h["wa"])
    ref = eng.solve_block(h["rho"], h["T"], h["dz"], fully_ionized_T=h["fully_ionized_T"], form="plain",
                          want=("Vtop", "Vbot"), allow_zero_pivot=True)
    eng.close()
    for k in ("Vtop", "Vbot"):
        assert np.array_equal(got[k].view(np.uint64), ref[k].view(np.uint64)), k
