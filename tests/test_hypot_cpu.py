"""The identity behind the GPU's complex column scan (k_hyp_z_pm): its magnitudes use the
project-own hypot with the power-of-two scalings done by IEEE multiplications where those
are exact, and fall back to the integer-SCALE form elsewhere.  On the CPU, with the same
IEEE operations, the two forms must agree bit for bit on every operand pair (oracle
jk_hypot_check.c: 2e7 seeded pairs from four distributions, including arbitrary bit
patterns, subnormals, infinities, NaNs and exponent gaps around 54).  The GPU parity tests
compare the kernel itself with the oracle."""
import oracle


def test_mulscaled_hypot_equals_scale_form():
    oracle.build()
    L = oracle.lib()
    assert L.jo_hypot_identity_check(20_000_000, 12345) == 0
    assert L.jo_hypot_identity_check(2_000_000, 777) == 0
