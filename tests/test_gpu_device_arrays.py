"""Per-site read-outs on the device (cacb200_device_array): the context's
arrays as torch CUDA tensors without a copy must hold exactly what the host
read-outs return; compute pe/atom and stress/atom of the reference
(compute_pe_atom.cpp, compute_stress_atom.cpp: -nktv2p x per-site virial, no
kinetic term) then follow on the device."""
import numpy as np
import pytest

from helpers import CASES, LJ, SKIN

pytestmark = pytest.mark.gpu

NKTV2P = 1.6021765e6


def test_device_arrays_equal_host_readouts(tmp_path):
    from cac_b200.api import ENERGY_ATOM, ENERGY_GLOBAL, VIRIAL_ATOM, VIRIAL_GLOBAL, CacB200Error, Engine
    s = CASES["tiny_lj"][0]()
    e = Engine(0)
    e.upload(s)
    e.pair_lj(*LJ)
    e.neighbor(SKIN, 10)
    e.setup()
    e.run_nve(7)
    with pytest.raises(CacB200Error):
        e.device_array("eatom")          # no per-site tally yet
    e.compute(ENERGY_GLOBAL | ENERGY_ATOM, VIRIAL_GLOBAL | VIRIAL_ATOM)
    x, v, nx, nv = e.state()
    f, nf, _ = e.forces()
    ev = e.energy()
    dev = {k: e.device_array(k).cpu().numpy() for k in Engine.ARRAYS}
    assert np.array_equal(dev["x"][:, :3], x)
    assert np.array_equal(dev["v"], v) and np.array_equal(dev["f"], f)
    assert np.array_equal(dev["nodex"].reshape(-1, 8, 3), nx) and np.array_equal(dev["nodev"].reshape(-1, 8, 3), nv)
    assert np.array_equal(dev["nodef"].reshape(-1, 8, 3), nf)
    assert np.array_equal(dev["eatom"], ev["eatom"]) and np.array_equal(dev["enode"].reshape(-1, 8), ev["enode"])
    assert np.array_equal(dev["vatom"], ev["vatom"])
    assert np.array_equal(dev["vnode"].reshape(-1, 8, 6), ev["vnode"])
    # stress/atom on the device, without a host copy of the virials
    stress = -NKTV2P * e.device_array("vatom")
    assert np.array_equal(stress.cpu().numpy(), -NKTV2P * ev["vatom"])
    e.close()


@pytest.mark.parametrize("nsteps", [1, 13])
def test_run_from_host_arrays_equals_set_run_get(nsteps):
    """cacb200_run_nve_host (state in, steps, state out, the position copy
    beside the last step's forces) gives what set_state + run_nve +
    get_state give, bit for bit, step after step (a list rebuild included)."""
    import torch
    from cac_b200.api import Engine
    s = CASES["tiny_lj"][0]()
    out = []
    for host in (True, False):
        e = Engine(0)
        e.upload(s)
        e.pair_lj(*LJ)
        e.neighbor(SKIN, 10)
        e.setup()
        x, v, nx, nv = (torch.from_numpy(a.copy()).pin_memory().numpy() for a in e.state())
        for _ in range(3):
            if host:
                e.run_nve_host(nsteps, x, v, nx, nv)
            else:
                e.set_state(x, v, nx, nv)
                e.run_nve(nsteps)
                x, v, nx, nv = e.state()
        out.append((x.copy(), v.copy(), nx.copy(), nv.copy()))
        e.close()
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)
