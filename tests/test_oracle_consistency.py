"""The oracle's forms that the reference does not have (trilinear slicing,
the poisson scaling update) checked against their mathematics on CPU:
trilinear weights at integer positions select one voxel, so trilinear and
nearest slices agree there; and the poisson update is the maximum of the
expected log-likelihood over the pattern's scale."""
import numpy as np


def test_trilinear_at_integer_positions_equals_nearest(orc):
    side, n_rot = 8, 3
    rng = np.random.default_rng(11)
    model = rng.uniform(0.1, 2.0, side ** 3)
    # identity rotations: position u = side/2 + 0.5 + c, so c = k - side/2 - 0.5
    # puts every pixel on voxel k exactly (in FP32 too: small dyadic values)
    k = rng.integers(1, side - 1, size=(3, side * side))
    cx, cy, cz = (k[i] - side / 2 - 0.5 for i in range(3))
    rot = np.tile(np.array([1.0, 0.0, 0.0, 0.0]), (n_rot, 1))
    near = orc.expand(orc.make_config(side, 1, n_rot, interp=orc.NEAREST), model, rot, cx, cy, cz)
    tri = orc.expand(orc.make_config(side, 1, n_rot, interp=orc.TRILINEAR), model, rot, cx, cy, cz)
    np.testing.assert_array_equal(tri, near)
    expect = model[(k[2] * side + k[1]) * side + k[0]]
    np.testing.assert_allclose(near[0], expect, rtol=1e-7)


def test_poisson_scaling_update_maximises_the_expected_loglik(orc):
    side, N, n_rot = 8, 5, 6
    rng = np.random.default_rng(12)
    npix = side * side
    S = rng.uniform(0.05, 1.5, (n_rot, npix))
    images = rng.poisson(2.0, (N, npix)).astype(np.float32)
    mask = np.ones(npix, np.int32)
    mask[:5] = 0  # masked pixels take no part
    P = rng.dirichlet(np.ones(n_rot), size=N).T  # [R][N], columns sum to 1
    cfg = orc.make_config(side, N, n_rot, likelihood=orc.LL_POISSON)
    phi = orc.update_scaling(cfg, S, images, mask, P, np.ones(N))
    act = mask != 0

    def Q(p, f):  # sum_r P_rp (sum_j K_j log(f W_rj) - f sum_j W_rj) over active pixels
        K = images[p, act].astype(np.float64)
        W = S[:, act]
        return float(np.sum(P[:, p] * ((np.log(f * W) * K).sum(1) - f * W.sum(1))))

    for p in range(N):
        q0 = Q(p, phi[p])
        for step in (1e-3, -1e-3):
            assert Q(p, phi[p] * (1 + step)) < q0
