"""Requests the device cannot serve end as status codes, and the device
stays usable: a simulation too large for device memory (the allocation
really fails), more particles than the slot tags allow, a grid with more
cells than 32-bit cell ids reach, and a device that does not exist.  After
each, a normal simulation on the same device still equals the oracle."""
import ctypes as C

import numpy as np
import pytest

import psb200
from psb200 import scenes
from oracle import ps_oracle as O

pytestmark = pytest.mark.gpu

PS_ERR_INVALID, PS_ERR_NOMEM = -1, -3


def create_raw(n_particles, precision=0, device=0):
    """ps_create on one box scene of n_particles with no state uploaded."""
    d = psb200.SceneDesc()
    d.n_particles = n_particles
    d.box_min = (C.c_double * 3)(0.0, 0.0, 0.0)
    d.box_max = (C.c_double * 3)(1.0, 1.0, 1.0)
    d.gravity = (C.c_double * 3)(0.0, 0.0, -9.8)
    d.e_wall = (C.c_double * 6)(*([0.8] * 6))
    d.k_spring, d.e_sphere, d.dt = 1.0, 0.5, 1e-5
    arr = (psb200.SceneDesc * 1)(d)
    h = C.c_void_p()
    rc = psb200.lib().ps_create(arr, 1, precision, device, C.byref(h))
    if rc == 0:
        psb200.lib().ps_destroy(h)
    return rc, psb200.lib().ps_last_error().decode()


def still_healthy():
    sc = scenes.pile(500, seed=8, k_spring=1.0)
    with psb200.Simulation(sc, "f32") as sim:
        sim.set_state()
        sim.step(20)
        got = sim.get_state().astype(np.float32)
    assert np.array_equal(got, O.run(sc, 20, "f32"))


@pytest.mark.parametrize("precision", [0, 1])
def test_simulation_larger_than_device_memory(need_gpu, precision):
    # 2^31 - 100 particles need more than 300 GB of particle arrays
    rc, msg = create_raw((1 << 31) - 100, precision)
    assert rc == PS_ERR_NOMEM and "ps_create" in msg, (rc, msg)
    still_healthy()


def test_more_particles_than_slot_tags_allow(need_gpu):
    rc, msg = create_raw(1 << 31)
    assert rc == PS_ERR_INVALID and "too many particles" in msg, (rc, msg)
    still_healthy()


def test_grid_with_more_cells_than_32_bit_ids(need_gpu):
    # radius 1e-3 in a box of edge 100: 47,620^3 cells
    sc = scenes.pile(64, seed=9).copy(box_min=(0.0, 0.0, 0.0), box_max=(100.0, 100.0, 100.0))
    sc.state[:, 6] = 1e-3
    with psb200.Simulation(sc, "f32") as sim:
        with pytest.raises(psb200.PSError, match="too many grid cells"):
            sim.set_state()
    still_healthy()


def test_device_that_does_not_exist(need_gpu):
    rc, msg = create_raw(100, 0, device=99)
    assert rc == PS_ERR_INVALID and "no CUDA device" in msg, (rc, msg)
    still_healthy()
