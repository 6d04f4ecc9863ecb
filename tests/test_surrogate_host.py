"""Host side of the photon surrogate (no GPU): argument validation of the
network, photon-beam and gamma entry points of the C ABI, the layer table and
FLOP count, the fragment packing size, and the phantom/field generator of the
surrogate workload."""
import ctypes as C

import numpy as np
import pytest
import torch

from dosecuda_b200 import _lib
from dosecuda_b200.surrogate import ARCH, LEVELS, SurrogateNet, hu_to_density, random_field, random_phantom_hu, \
    weight_shape

V = C.c_void_p


def test_architecture_is_a_four_level_encoder_decoder():
    chans = sorted({c for _, _, ci, co in ARCH for c in (ci, co) if c >= 16})
    assert tuple(chans) == LEVELS == (16, 32, 64, 128)
    kinds = [k for _, k, _, _ in ARCH]
    assert kinds.count("down") == 3 and kinds.count("up") == 3
    assert ARCH[0][2] == 8 and ARCH[-1][3] == 16  # padded 2-channel input; 16 features into the head
    # encoder and decoder mirror each other
    assert [c for _, k, _, c in ARCH if k == "down"] == [32, 64, 128]
    assert [c for _, k, _, c in ARCH if k == "up"] == [64, 32, 16]


def test_flop_count_from_layer_shapes():
    d = h = w = 128
    v0 = d * h * w
    expect = 0
    expect += 2 * v0 * 16 * 8 * 27            # enc0
    expect += 2 * (v0 // 8) * 32 * 16 * 8     # down0
    expect += 2 * (v0 // 8) * 32 * 32 * 27    # enc1
    expect += 2 * (v0 // 64) * 64 * 32 * 8    # down1
    expect += 2 * (v0 // 64) * 64 * 64 * 27   # enc2
    expect += 2 * (v0 // 512) * 128 * 64 * 8  # down2
    expect += 2 * (v0 // 512) * 128 * 128 * 27  # bottleneck
    expect += 2 * (v0 // 64) * 64 * 128       # up2
    expect += 2 * (v0 // 64) * 64 * 64 * 27   # dec2
    expect += 2 * (v0 // 8) * 32 * 64         # up1
    expect += 2 * (v0 // 8) * 32 * 32 * 27    # dec1
    expect += 2 * v0 * 16 * 32                # up0
    expect += 2 * v0 * 16 * 16 * 27           # dec0
    expect += 2 * v0 * 16                     # head
    assert SurrogateNet.flops((d, h, w)) == expect
    assert 90e9 < expect < 110e9


def test_packed_fragment_sizes():
    lib = _lib.load()
    assert lib.dc_net_packed_fragments(27, 16, 16) == 27 * 16 // 16 * 2 * 32
    assert lib.dc_net_packed_fragments(27, 8, 16) == 14 * 2 * 32  # 216 k-rows -> 14 k16 steps
    assert lib.dc_net_packed_fragments(8, 128, 64) == 64 * 8 * 32
    assert lib.dc_net_packed_fragments(27, 16, 12) == -1  # n must be a multiple of 8
    for name, kind, cin, cout in ARCH:
        shp = weight_shape(kind, cin, cout)
        assert shp == ((8, cout, cin) if kind == "up" else ((27 if kind == "conv3" else 8), cin, cout))


def test_net_entry_points_validate_before_touching_a_gpu():
    lib = _lib.load()
    x = np.zeros(64, np.uint16)
    p = x.ctypes.data_as(V)
    s = None
    # unsupported channel pair
    assert lib.dc_net_conv(0, 0, p, 1, 4, 4, 4, 24, p, 10, 24, p, None, s) == _lib.DC_ERR_VALUE
    assert "unsupported" in lib.dc_last_error().decode()
    # packed weights of the wrong size
    assert lib.dc_net_conv(0, 0, p, 1, 4, 4, 4, 16, p, 10, 16, p, None, s) == _lib.DC_ERR_VALUE
    assert "packed weights" in lib.dc_last_error().decode()
    # odd grid for the stride-2 convolution
    assert lib.dc_net_conv(0, 1, p, 1, 3, 4, 4, 16, p, 8 * 2 * 4 * 32, 32, p, None, s) == _lib.DC_ERR_VALUE
    # NULL buffers
    assert lib.dc_net_conv(0, 0, None, 1, 4, 4, 4, 16, p, 27 * 2 * 32, 16, p, None, s) == _lib.DC_ERR_VALUE
    assert lib.dc_net_conv_up(0, p, 1, 2, 2, 2, 48, p, 1, 24, None, p, s) == _lib.DC_ERR_VALUE
    assert lib.dc_net_wgrad(0, 0, p, p, 1, 4, 4, 4, 24, 24, p, s) == _lib.DC_ERR_VALUE
    assert lib.dc_net_norm_act(0, p, 1, 8, 12, p, 0.01, p, s) == _lib.DC_ERR_VALUE
    assert lib.dc_net_head(0, p, 8, 32, p, p, p, 0.0, 1.0, p, s) == _lib.DC_ERR_VALUE
    assert lib.dc_net_pack_weights(0, p, 27, 16, 12, 0, 0, p, s) == _lib.DC_ERR_VALUE


def test_photon_beam_and_gamma_validate_before_touching_a_gpu():
    lib = _lib.load()
    h = C.c_void_p()
    assert lib.dc_photon_beam_create(0, 0, 4, 4, _lib.f3((1, 1, 1)), _lib.f3((0, 0, 0)), C.byref(h)) == \
        _lib.DC_ERR_VALUE
    assert lib.dc_photon_beam_create(0, 4, 4, 4, _lib.f3((1, -1, 1)), _lib.f3((0, 0, 0)), C.byref(h)) == \
        _lib.DC_ERR_VALUE
    assert not h.value
    x = np.zeros(64, np.float32)
    p = x.ctypes.data_as(V)
    assert lib.dc_photon_beam_dose(None, p, None) == _lib.DC_ERR_VALUE
    assert lib.dc_photon_beam_probe(None, None, 0, p, None) == _lib.DC_ERR_VALUE
    assert lib.dc_gamma(0, p, 4, 4, 4, _lib.f3((1, 1, 1)), None, p, 0, 0.0, 0.0, 0.02, 0.1, p, None) == \
        _lib.DC_ERR_VALUE  # dta must be positive
    assert lib.dc_gamma(0, None, 4, 4, 4, _lib.f3((1, 1, 1)), None, p, 0, 0.0, 2.0, 0.02, 0.1, p, None) == \
        _lib.DC_ERR_VALUE


def test_hu_to_density_is_np_interp():
    from dosecuda_b200.lookup import table_path
    import pandas as pd
    df = pd.read_csv(table_path("photons", "VarianTrueBeamHF", "HU_Density.csv"))
    hu = torch.linspace(-1500.0, 4000.0, 1001)
    got = hu_to_density(hu, df["HU"].to_numpy(), df["Density"].to_numpy()).numpy()
    ref = np.interp(hu.numpy().astype(np.float64), df["HU"].to_numpy(), df["Density"].to_numpy())
    np.testing.assert_allclose(got, ref.astype(np.float32), rtol=1e-6, atol=1e-6)


def test_surrogate_phantoms_and_fields():
    rng = np.random.default_rng(3)
    hu = random_phantom_hu(rng, (32, 32, 32), 10.0, device="cpu")
    assert hu.shape == (32, 32, 32)
    assert float(hu.min()) >= -1000.0 and float(hu.max()) <= 1500.0
    assert float((hu == -1000.0).float().mean()) > 0.2  # air around the body
    assert float((hu == 0.0).float().mean()) > 0.05     # water body
    inside = hu[(hu > -1000.0) & (hu != 0.0)]
    assert inside.numel() > 0 and float(inside.min()) >= -900.0
    # the same seed gives the same phantom
    hu2 = random_phantom_hu(np.random.default_rng(3), (32, 32, 32), 10.0, device="cpu")
    assert torch.equal(hu, hu2)
    gantries, sides = [], []
    r = np.random.default_rng(0)
    for _ in range(400):
        g, fx, fy = random_field(r)
        gantries.append(g)
        sides += [fx, fy]
    assert all(g % 5.0 == 0.0 and 0.0 <= g < 360.0 for g in gantries)
    assert len(set(gantries)) > 50
    assert 2.0 <= min(sides) and max(sides) <= 20.0


def test_tensor_core_conv_validates_before_touching_a_gpu():
    lib = _lib.load()
    x = np.zeros(64, np.uint16)
    p = x.ctypes.data_as(V)
    assert lib.dc_net_packed_tc_bytes(16, 16) == 27 * 2 * 16 * 16
    assert lib.dc_net_packed_tc_bytes(8, 16) == 18 * 2 * 16 * 16
    assert lib.dc_net_packed_tc_bytes(32, 32) == -1
    nb = lib.dc_net_packed_tc_bytes(16, 16)
    # x extent must be 128, y/z even
    assert lib.dc_net_conv_tc(0, p, 1, 4, 4, 64, 16, p, nb, 16, p, None, None) == _lib.DC_ERR_VALUE
    assert lib.dc_net_conv_tc(0, p, 1, 3, 4, 128, 16, p, nb, 16, p, None, None) == _lib.DC_ERR_VALUE
    assert "x extent 128" in lib.dc_last_error().decode()
    # packed size must match
    assert lib.dc_net_conv_tc(0, p, 1, 4, 4, 128, 16, p, nb - 16, 16, p, None, None) == _lib.DC_ERR_VALUE
    assert lib.dc_net_pack_weights_tc(0, p, 8, 16, 16, 0, 0, p, None) == _lib.DC_ERR_VALUE


def test_hu_table_validation_before_touching_a_gpu():
    lib = _lib.load()
    x = np.zeros(64, np.float32)
    p = x.ctypes.data_as(V)
    th = np.array([-1000.0, 0.0, 0.0, 1000.0])  # not strictly increasing
    tv = np.array([0.0, 1.0, 1.0, 2.0])
    assert lib.dc_hu_convert_dev(0, p, 2, 2, 2, th.ctypes.data_as(V), tv.ctypes.data_as(V), 4, p, None) == \
        _lib.DC_ERR_VALUE
    assert "increasing" in lib.dc_last_error().decode()
    th2 = np.linspace(-1000.0, 3000.0, 65)
    tv2 = np.ones(65)
    assert lib.dc_hu_convert_dev(0, p, 2, 2, 2, th2.ctypes.data_as(V), tv2.ctypes.data_as(V), 65, p, None) == \
        _lib.DC_ERR_VALUE


def test_texture_calibration_validates_before_touching_a_gpu():
    assert _lib.load().dc_texture_fetch_rate(0, None) == _lib.DC_ERR_VALUE
