"""The identity the fast insertion kernel uses for the hull in-circle test of a
set whose filters are exact (build.cu, hull_in_circle_ex): for a point p in the
plane of the hull facet (a, b, d) and the apex x of the finite tet across it,

    sign in_circle(a, b, d, p) = sign det_in_sphere(a, b, d, x, p) * sign det_orient3d(a, b, d, x)

with each determinant written as the device filters write it (predicates.cuh:
orient3d_filter, in_sphere_filter, in_circle_filter; the reference's
src/predicates.cpp:125-204 and src/predicates2.cpp:182-231), evaluated here in
exact integer arithmetic on random coplanar lattice configurations.  The
in-circle value is zero exactly when the in-sphere value is, so the cocircular
tie-break is reached in the same cases."""
import random

import pytest


def sgn(v):
    return (v > 0) - (v < 0)


def orient_det(a, b, c, d):
    adx, bdx, cdx = a[0] - d[0], b[0] - d[0], c[0] - d[0]
    ady, bdy, cdy = a[1] - d[1], b[1] - d[1], c[1] - d[1]
    adz, bdz, cdz = a[2] - d[2], b[2] - d[2], c[2] - d[2]
    return adz * (bdx * cdy - cdx * bdy) + bdz * (cdx * ady - adx * cdy) + cdz * (adx * bdy - bdx * ady)


def insphere_det(a, b, c, d, e):
    aex, aey, aez = (a[i] - e[i] for i in range(3))
    bex, bey, bez = (b[i] - e[i] for i in range(3))
    cex, cey, cez = (c[i] - e[i] for i in range(3))
    dex, dey, dez = (d[i] - e[i] for i in range(3))
    ab, bc, cd = aex * bey - bex * aey, bex * cey - cex * bey, cex * dey - dex * cey
    da, ac, bd = dex * aey - aex * dey, aex * cey - cex * aey, bex * dey - dex * bey
    abc = aez * bc - bez * ac + cez * ab
    bcd = bez * cd - cez * bd + dez * bc
    cda = cez * da + dez * ac + aez * cd
    dab = dez * ab + aez * bd + bez * da
    al = aex * aex + aey * aey + aez * aez
    bl = bex * bex + bey * bey + bez * bez
    cl = cex * cex + cey * cey + cez * cez
    dl = dex * dex + dey * dey + dez * dez
    return (dl * abc - cl * dab) + (bl * cda - al * bcd)


def incircle_det(p0, p1, p2, p):
    pt = [p0[i] - p[i] for i in range(3)]
    qt = [p1[i] - p[i] for i in range(3)]
    rt = [p2[i] - p[i] for i in range(3)]
    pq = [p1[i] - p0[i] for i in range(3)]
    pr = [p2[i] - p0[i] for i in range(3)]
    vx = pq[1] * pr[2] - pq[2] * pr[1]
    vy = pq[2] * pr[0] - pq[0] * pr[2]
    vz = pq[0] * pr[1] - pq[1] * pr[0]
    a00, a01, a02, a03 = pt[0], pt[1], pt[2], sum(x * x for x in pt)
    a10, a11, a12, a13 = rt[0], rt[1], rt[2], sum(x * x for x in rt)
    a20, a21, a22, a23 = qt[0], qt[1], qt[2], sum(x * x for x in qt)
    a30, a31, a32, a33 = vx, vy, vz, vx * vx + vy * vy + vz * vz
    m01, m02, m03 = a10 * a01 - a00 * a11, a20 * a01 - a00 * a21, a30 * a01 - a00 * a31
    m12, m13, m23 = a20 * a11 - a10 * a21, a30 * a11 - a10 * a31, a30 * a21 - a20 * a31
    m012 = m12 * a02 - m02 * a12 + m01 * a22
    m013 = m13 * a02 - m03 * a12 + m01 * a32
    m023 = m23 * a02 - m03 * a22 + m02 * a32
    m123 = m23 * a12 - m13 * a22 + m12 * a32
    return m123 * a03 - m023 * a13 + m013 * a23 - m012 * a33


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_lifted_in_circle_matches_in_circle(seed):
    rng = random.Random(seed)
    checked = zeros = 0
    while checked < 6000:
        o = [rng.randint(-20, 20) for _ in range(3)]
        u = [rng.randint(-6, 6) for _ in range(3)]
        w = [rng.randint(-6, 6) for _ in range(3)]

        def plane(s, t):
            return [o[i] + s * u[i] + t * w[i] for i in range(3)]

        a, b, d, p = (plane(rng.randint(-4, 4), rng.randint(-4, 4)) for _ in range(4))
        if len({tuple(a), tuple(b), tuple(d), tuple(p)}) < 4:
            continue
        x = [rng.randint(-25, 25) for _ in range(3)]
        ox = orient_det(a, b, d, x)
        if ox == 0:
            continue   # a, b, d collinear, or x in their plane: not a tet
        assert orient_det(a, b, d, p) == 0
        ic = sgn(incircle_det(a, b, d, p))
        lifted = sgn(insphere_det(a, b, d, x, p)) * sgn(ox)
        assert ic == lifted, (a, b, d, p, x)
        zeros += ic == 0
        checked += 1
    assert zeros > 0   # the cocircular case was reached
