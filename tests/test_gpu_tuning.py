"""GPU tests of the tuned launch parameters and the autotuner: every
candidate setting gives the same counts; the tuner keeps them exact."""
import itertools

import numpy as np
import pytest

import signed_triangle_counting_b200 as stc

from test_gpu_dispatch import clique_counts

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def clique():
    # K_1300: out-degrees 0..1299 in rank space, so warp, block and large
    # lists all occur.
    k = 1300
    rng = np.random.default_rng(77)
    a, b = np.triu_indices(k, 1)
    s = np.where(rng.random(len(a)) < 0.55, 1, -1).astype(np.int8)
    S = np.zeros((k, k), np.int8)
    S[a, b] = s
    S[b, a] = s
    perm = rng.permutation(k).astype(np.uint32)
    return perm[a], perm[b], s, clique_counts(S)


def test_every_candidate_is_exact(ctx, clique):
    src, dst, sign, want = clique
    for bt, hf, u in itertools.product((128, 256, 512), (2, 4, 8), (1, 2, 4)):
        t = {"block_threads": bt, "hash_factor": [hf, hf, min(hf, 4)], "unroll": [u, u, u]}
        ctx.set_tuning(t)
        assert ctx.get_tuning() == t
        assert ctx.count(src, dst, sign).as_tuple() == want, t
    ctx.set_tuning(None)


def test_autotune_keeps_counts(ctx, clique):
    src, dst, sign, want = clique
    t = ctx.autotune(src, dst, sign, reps=1)
    assert t["block_threads"] in (128, 256, 512)
    assert ctx.get_tuning() == t
    assert ctx.count(src, dst, sign).as_tuple() == want
    ctx.set_tuning(None)
    assert ctx.get_tuning() == {"block_threads": 256, "hash_factor": [4, 4, 2], "unroll": [2, 2, 2]}


def test_invalid_tuning_rejected(ctx):
    for bad in ({"block_threads": 64, "hash_factor": [4, 4, 2], "unroll": [2, 2, 2]},
                {"block_threads": 256, "hash_factor": [3, 4, 2], "unroll": [2, 2, 2]},
                {"block_threads": 256, "hash_factor": [4, 4, 2], "unroll": [2, 8, 2]}):
        with pytest.raises(stc.StcError):
            ctx.set_tuning(bad)


def test_shipped_tuning_loads(ctx):
    from signed_triangle_counting_b200 import autotune
    for w in ("2", "3", "4", "5"):
        t = autotune.tuning_for(int(w))
        assert t is not None, w
        ctx.set_tuning(t)
    ctx.set_tuning(None)
