"""Host logic of the drop-in kernel's learned tuner (no GPU)."""


def test_reference_space_is_the_reference_enumeration():
    """The drop-in tuner's "reference" space is every shape of the reference's sweep
    (cuda/primes.cpp): 464 in 2D and 2,723 in 3D at 1024 threads, the power-of-two space inside it."""
    from threadcoarsenedstencilgenerator_b200 import autotune as A

    for d, n in ((2, 464), (3, 2723)):
        ref = A.blocks_of("reference", d)
        assert len(ref) == n == len(set(ref))
        assert set(A.blocks_of("pow2", d)) <= set(ref)
        assert all(b[0] * b[1] * b[2] <= 1024 for b in ref)
