"""Host logic of the chunked host-buffer calls (no GPU needed):
sdg_rk3_steps_host and sdg_cal_tend cut the element range into chunks and
launch each RK stage chunk by chunk as its inputs arrive.

The chunk boundaries put one reach (a z-layer in a periodic box) into each
of the three first and four last chunks, the band that can only finish
after the last upload.  The launch plan must respect every dependency
(stage g of chunk j after stage g-1 of its neighbour chunks; stage 0 after
their uploads), cover every (stage, chunk) once, and overwrite no chunk's
q0 (stage 3) before every chunk that reads it in stage 1 has run; the GPU
tests check the results bit for bit, these the schedule itself.
"""
import numpy as np
import pytest

import sdg_b200 as sdg


@pytest.fixture(scope="module", autouse=True)
def _build(built):
    return built


def ring(S):
    """Neighbour lists of z-layer chunks of a periodic box (reach-thick
    chunks or thicker): the chunk itself and the chunks before and after."""
    return [sorted({(j - 1) % S, j, (j + 1) % S}) for j in range(S)]


@pytest.mark.parametrize("Ne,Np,reach,S", [
    (32768, 512, 1024, 20),    # 32^3 p = 7: thin ends of one z-layer
    (4096, 4096, 256, 16),     # 16^3 p = 15
    (8192, 64, 256, 16),       # thin chunks of 512 elements (the smallest)
    (4096, 64, 256, 8),        # too few elements for thin ends: 8 equal
    (2048, 1000, 64, 7),       # p = 9: chunks of >= 262 elements
    (64, 64, 16, 0),           # too small to pipeline
])
def test_chunk_bounds(Ne, Np, reach, S):
    e0 = sdg.chunk_bounds(Ne, Np, reach)
    assert len(e0) == (S + 1 if S else 0)
    if not S:
        return
    assert e0[0] == 0 and e0[-1] == Ne
    size = np.diff(e0)
    assert (size > 0).all()
    assert (size >= min(512, (1 << 18) // Np)).all()
    if S == 20 or (S == 16 and Ne >= 9 * max(reach, min(512, (1 << 18) // Np))):
        thin = max(reach, min(512, (1 << 18) // Np))
        assert (size[:3] == thin).all() and (size[-4:] == thin).all()


def simulate(plan, nbr, uploads, steps=1):
    """Checks every dependency of the plan; returns the chunks whose last
    stage runs after the wait for the last upload."""
    S, G = len(nbr), 3 * steps
    done = np.zeros((G, S), dtype=bool)
    waited = -1
    late = []
    for g, j0, j1, need in plan:
        assert 0 <= g < G and 0 <= j0 <= j1 < S
        waited = max(waited, need)
        for j in range(j0, j1 + 1):
            assert not done[g, j], "launched twice"
            for c in nbr[j]:
                if g == 0:
                    assert not uploads or c <= waited, "reads a chunk not yet uploaded"
                else:
                    assert done[g - 1, c], "reads a stage input not yet written"
            if g >= 2:
                # Stage g overwrites a buffer (q0 for g % 3 == 2, else the
                # output of stage g - 3) that stage g - 2 of every chunk
                # whose list holds j reads: all of them have run.
                for k in range(S):
                    if j in nbr[k]:
                        assert done[g - 2, k], "overwrites a buffer still to be read"
            if g == G - 1 and uploads and waited == S - 1:
                late.append(j)
        done[g, j0:j1 + 1] = True
    assert done.all()
    return late


@pytest.mark.parametrize("S,steps", [(4, 1), (5, 1), (8, 1), (16, 1), (20, 1),
                                     (20, 2), (20, 3), (8, 3)])
def test_step_plan_with_uploads(S, steps):
    nbr = ring(S)
    plan = sdg.step_plan(nbr, uploads=True, steps=steps)
    late = simulate(plan, nbr, True, steps)
    # The last upload's chunk and its neighbours to a depth of three a step.
    r = 3 * steps
    assert sorted(late) == sorted({j % S for j in range(S - 1 - r, S + r)})
    # Stage 0 waits for the uploads in chunk order.
    needs = [n for g, _, _, n in plan if g == 0]
    assert needs == sorted(needs)
    # Only the tail merges: the launches before the wait for the last
    # upload hold one chunk each.
    first_last = next(i for i, (g, _, _, n) in enumerate(plan) if n == S - 1)
    assert all(j0 == j1 for _, j0, j1, _ in plan[:first_last])


@pytest.mark.parametrize("S", [4, 16, 20])
def test_step_plan_without_uploads_stays_per_chunk(S):
    """The last step of a multi-step call: no uploads, one launch per
    (stage, chunk), so that the state's chunks go back as they finish."""
    nbr = ring(S)
    plan = sdg.step_plan(nbr, uploads=False)
    simulate(plan, nbr, False)
    assert len(plan) == 3 * S
    assert (plan[:, 3] == -1).all()
    # With more than a few chunks, the first stage 3 (and its download)
    # comes well before the end.
    first_s3 = next(i for i, row in enumerate(plan) if row[0] == 2)
    if S >= 8:
        assert first_s3 < len(plan) // 2


def test_step_plan_general_neighbours():
    """A non-ring relation (chunks that also touch the chunk two away) still
    yields a valid plan."""
    S = 10
    nbr = [sorted({(j + d) % S for d in (-2, -1, 0, 1, 2)}) for j in range(S)]
    for uploads in (True, False):
        simulate(sdg.step_plan(nbr, uploads), nbr, uploads)


def test_step_plan_rejects_bad_lists():
    with pytest.raises(sdg.SdgError) as e:
        sdg.step_plan([[0, 1], [0, 5]], uploads=True)
    assert e.value.code == sdg.SDG_ERR_ARG


def test_chunk_bounds_rejects_bad_arguments():
    for args in ((0, 64, 1), (64, 0, 1), (64, 64, 0), (64, 64, 65)):
        with pytest.raises(sdg.SdgError) as e:
            sdg.chunk_bounds(*args)
        assert e.value.code == sdg.SDG_ERR_ARG
