"""Host parameter search: the minimum-root rule against the reference's pinned OpenFHE table."""
from ntt_gpu_b200.params import find_psi, min_psi
from oracle.oracle import PINNED_N, PINNED_P, PINNED_P_PSI, PINNED_Q, PINNED_Q_PSI


def test_min_psi_reproduces_the_pinned_openfhe_roots():
    for q, psi in zip(PINNED_Q + PINNED_P, PINNED_Q_PSI + PINNED_P_PSI):
        assert min_psi(q, PINNED_N) == psi


def test_min_psi_is_a_primitive_root_no_larger_than_find_psi():
    q = 1152921504606584833
    for n in (1024, 4096):
        r = min_psi(q, n)
        assert pow(r, n, q) == q - 1
        assert r <= find_psi(q, n)
