"""XSalsa20 keystream and samplers on the B200 vs the oracle."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def test_xsalsa20_stream():
    from kunpbfv_b200.api import salsa20_stream
    rng = np.random.default_rng(1)
    for nbytes, block0 in [(64, 0), (1000, 0), (4096, 7)]:
        key = bytes(rng.integers(0, 256, 32, dtype=np.uint8))
        nonce = bytes(rng.integers(0, 256, 24, dtype=np.uint8))
        got = salsa20_stream(key, nonce, nbytes, block0).cpu().numpy().tobytes()
        assert got == oracle.xsalsa20(key, nonce, nbytes, block0)


def test_reference_compat_stream():
    """The reference's VecCrypt variant (zero sigma, 32-bit nonce, tail left zero)."""
    from kunpbfv_b200.api import salsa20_stream
    key = bytes(range(32))
    nonce = (0x1234567).to_bytes(4, "little") + b"\x00" * 20
    for nbytes in (128, 200):
        got = salsa20_stream(key, nonce, nbytes, compat=True).cpu().numpy().tobytes()
        assert got == oracle.salsa20_compat(key, 0x1234567, nbytes)
