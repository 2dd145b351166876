"""Host logic of the post-processing modules and the export, on a stub
solver (no GPU): dataset names, the calls each module makes (export
dimensions passed to the device-side resize, far-field parameters), the
uint8 scalings of post::IntensityUint8 / LogIntensityUint8
(src/postProcessMod.cpp:17-84), the group and far-field attributes
(src/paraxialSimulation.cpp:453-510, src/farFieldPost.cpp:131-139)."""
import json
import math
import os
from types import SimpleNamespace

import numpy as np

from paxpro_b200 import _capi, post


class StubSolver:
    """Records the calls a module makes; returns fixed arrays."""

    def __init__(self, three_d=True):
        self.three_d = three_d
        self.calls = []
        d = SimpleNamespace(min=-1.0, max=1.0, step=0.5)
        self.spec = SimpleNamespace(x=d, y=d, z=SimpleNamespace(min=0.0, max=4.0, step=1.0),
                                    wavenumber=40.0, kind=_capi.FFT_SOLVER_3D)
        self.save_n = 4
        self._u0_host = None

    def get_post(self, q, slot=-1):
        self.calls.append(("post", q, slot))
        return np.full((4, 4), float(q + 1))

    def get_post_resized(self, q, rows, cols, slot=-1):
        self.calls.append(("resized", q, rows, cols))
        return np.full((rows, cols), float(q + 1))

    def farfield(self, **kw):
        self.calls.append(("farfield", kw))
        return np.ones((3, 5))

    def num_saved(self):
        return 2


def test_projection_modules_resize_on_the_device_when_asked():
    s = StubSolver()
    ei = post.ExitIntensity()
    assert ei.result(s).shape == (4, 4) and s.calls[-1] == ("post", _capi.POST_ABS2, -1)
    ei.set_export_dimensions(2, 3)
    assert ei.result(s).shape == (2, 3)
    assert s.calls[-1] == ("resized", _capi.POST_ABS2, 2, 3)


def test_farfield_module_parameters_and_attributes():
    s = StubSolver()
    ff = post.FarField(pad_length=1024, phi_min=-0.5, phi_max=0.5, subtract_reference=True)
    ff.set_export_dimensions(64, 64)
    assert ff.result(s).shape == (3, 5)
    kw = s.calls[-1][1]
    assert kw["pad_length"] == 1024 and kw["phi_min"] == -0.5 and kw["phi_max"] == 0.5
    assert kw["export_dims"] == (64, 64) and kw["subtract_reference"] is True
    a = ff.attributes(s)
    assert a["qmax"] == 0.5 * 40.0 * math.pi / 180.0 and a["phiMin"] == -0.5


def test_uint8_scalings():
    s = StubSolver()
    s.get_post = lambda q, slot=-1: np.array([[0.5, 1.0], [2.0, 4.0]])
    u8 = post.IntensityUint8().result(s)
    assert u8.dtype == np.uint8
    assert list(u8[..., 0].ravel(order="F")) == [31, 127, 63, 255]   # trunc(255 a / max)
    lg = post.LogIntensityUint8()
    lg.set_min_value(1.0)
    out = lg.result(s)[..., 0]
    # log(0.5) < log(1) = min: clamped to 0; max log(4) -> 255
    assert out[0, 0] == 0 and out[1, 1] == 255
    assert out[0, 1] == 0                      # log(1) = min
    assert out[1, 0] == math.trunc(255.0 * (math.log(2.0) - 0.0) / (math.log(4.0) - 0.0))


def test_save_writes_named_datasets_and_attributes(tmp_path):
    s = StubSolver()
    mods = [post.ExitField(), post.ExitPhase(), post.FarField(pad_length=256)]
    written = post.save(s, str(tmp_path), mods, description="stub")
    names = sorted(os.path.basename(w) for w in written)
    assert names == ["exitField.npy", "exitPhase.npy", "farField.npy"]
    arr = np.load(os.path.join(str(tmp_path), "data", "exitField.npy"))
    assert arr.flags["F_CONTIGUOUS"] and arr.shape == (4, 4)
    with open(os.path.join(str(tmp_path), "data", "attributes.json")) as fh:
        attrs = json.load(fh)
    assert attrs["description"] == "stub" and attrs["solver"] == "FFTSolver3D"
    assert attrs["dx"] == 0.5 and attrs["wavenumber"] == 40.0
    assert set(attrs["farField"]) == {"phiMin", "phiMax", "qmin", "qmax"}
