"""The oracle's e4m3 encoder (OCP 8-bit floating point, E4M3: bias 7, no
infinities, largest finite 448, subnormals k * 2^-9) against facts of the
format: exact values, ties to the even code, saturation, sign symmetry."""
import numpy as np


def test_e4m3_known_values(oracle):
    L = oracle.lib()
    enc, dec = L.dgo_e4m3_encode, L.dgo_e4m3_decode
    cases = {0.0: 0x00, 1.0: 0x38, 448.0: 0x7E, 2.0 ** -9: 0x01, 2.0 ** -6: 0x08, 240.0: 0x77, 256.0: 0x78,
             0.875 * 2.0 ** -6: 0x07}
    for x, c in cases.items():
        assert enc(x) == c, (x, hex(enc(x)))
        assert dec(c) == x
    assert enc(1e6) == 0x7E and enc(-1e6) == 0xFE  # saturating
    assert enc(1.0625) == 0x38 and enc(1.1875) == 0x3A  # ties to the even code
    assert enc(248.0) == 0x78 and enc(1.5 * 2.0 ** -9) == 0x02
    assert enc(-3.3) == 0x80 | enc(3.3)


def test_e4m3_round_trip_is_nearest(oracle):
    L = oracle.lib()
    vals = np.array([L.dgo_e4m3_decode(c) for c in range(0x7F)], dtype=np.float64)
    assert np.all(np.diff(vals) > 0)  # positive codes are increasing
    rng = np.random.default_rng(0)
    for x in rng.uniform(0, 460, 2000).astype(np.float32):
        c = L.dgo_e4m3_encode(float(x))
        best = np.min(np.abs(vals - x))
        assert abs(L.dgo_e4m3_decode(c) - float(x)) <= best + 1e-12


def test_fp8_encode_scales(oracle):
    X = np.array([[0.0, 1.0, -2.0, 255.0], [0.0, 0.0, 0.0, 0.0]], dtype=np.float32)
    codes, scales = oracle.fp8_encode(X)
    assert scales[0] == np.float32(255.0) / np.float32(448.0) and scales[1] == 1.0
    assert codes[0, 3] == 0x7E and codes[1].tolist() == [0, 0, 0, 0]
