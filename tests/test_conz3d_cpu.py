"""Host logic of Model.conz3d, the Python form of shygpu_conz3d: the
arguments reach the C-ABI in conz3d_omp's order (concentration_omp.f90:65-76,
with the model and basin in front), and arrays that the call would write
through or misread are refused before the library is called."""
import numpy as np
import pytest

import shygpu
from shygpu import cases


class FakeLib:
    def __init__(self):
        self.calls = []

    def shygpu_conz3d(self, *args):
        self.calls.append(args)
        return 0


def bare_model(case):
    m = shygpu.Model.__new__(shygpu.Model)      # no device: the call itself is faked
    m.h, m.cases, m._closed = 77, [case], True
    return m


@pytest.fixture
def setup(monkeypatch):
    c = cases.lagoon_case(nkn_target=300, nlv=4, ntracer=1)
    fake = FakeLib()
    monkeypatch.setattr(shygpu, "lib", lambda: fake)
    nkn, nel, nlv = c["nkn"], c["nel"], c["nlv"]
    a = dict(cn1=np.zeros((nkn, nlv), np.float32), difhv=np.ones((nel, nlv), np.float32),
             difv=np.zeros((nkn, nlv + 1), np.float32), cobs=np.ones((nkn, nlv), np.float32),
             rtauv=np.ones((nkn, nlv), np.float32), wsinkv=np.ones((nkn, nlv + 1), np.float32),
             load=np.ones((nkn, nlv), np.float32))
    return c, fake, a


def test_arguments_reach_the_abi_in_the_reference_order(setup):
    c, fake, a = setup
    m = bare_model(c)
    m.conz3d(0, a["cn1"], 30.0, 0.2, a["difhv"], a["difv"], 1e-6, 0.5, 1.0, 0.0, 3, 2, itvd=0, itvdv=0,
             cobs=a["cobs"], robs=1.0, rtauv=a["rtauv"], wsink=2.0, wsinkv=a["wsinkv"], rload=3.0,
             load=a["load"])
    (args,) = fake.calls
    assert len(args) == 28
    assert args[0] == 77 and args[1] == 0
    assert args[2] == a["cn1"].ctypes.data and args[3] is None            # cn1, co1
    assert args[4:6] == (30.0, 0.2)                                      # ddt, rkpar
    assert args[6] == a["difhv"].ctypes.data and args[7] == a["difv"].ctypes.data
    assert args[8] == 1e-6 and args[9] is None                           # difmol, cbound
    assert args[10:14] == (0, 0, None, None)                             # itvd, itvdv, gradxv, gradyv
    assert args[14] == a["cobs"].ctypes.data and args[15] == 1.0         # cobs, robs
    assert args[16] == a["rtauv"].ctypes.data and args[17] == 2.0        # rtauv, wsink
    assert args[18] == a["wsinkv"].ctypes.data and args[19] == 3.0       # wsinkv, rload
    assert args[20] == a["load"].ctypes.data                             # load
    assert args[21:24] == (0.5, 1.0, 0.0)                                # azpar, adpar, aapar
    assert args[24:] == (3, 2, c["nlv"], c["nlv"])                       # istot, isact, nlvddi, nlev


@pytest.mark.parametrize("bad", ["cn1_f64", "load_strided", "wsinkv_shape"])
def test_arrays_it_would_write_or_misread_are_refused(setup, bad):
    c, fake, a = setup
    if bad == "cn1_f64":
        a["cn1"] = a["cn1"].astype(np.float64)
    elif bad == "load_strided":
        a["load"] = np.ones((c["nkn"], 2 * c["nlv"]), np.float32)[:, ::2]
    else:
        a["wsinkv"] = np.ones((c["nkn"], c["nlv"]), np.float32)
    m = bare_model(c)
    with pytest.raises(ValueError):
        m.conz3d(0, a["cn1"], 30.0, 0.2, a["difhv"], a["difv"], 1e-6, 0.5, 1.0, 0.0, 1, 1,
                 wsink=1.0, wsinkv=a["wsinkv"], rload=1.0, load=a["load"])
    assert fake.calls == []
