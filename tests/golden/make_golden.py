"""Writes tests/golden/known_answers.json: small hand-constructed catalogues
with answers derived here from geometry and IEEE double arithmetic, written
out explicitly (no oracle and no library involved).

Cases
  equilateral   triangle of side 5 (all galaxies, unit weights), rmin 1,
                rmax 10, 3 bins: every pair in bin 2 (t = 4/3), the triangle
                in configuration (2,2,2) = rank 7 of the 10 ordered triples.
  collinear     points at x = 0, 3, 4, 7, 10, 11: separations that land
                exactly on bin edges (t = 1.0 and 2.0 after IEEE rounding of
                (d - rmin) * fl(1/3)), on rmin (excluded) and on rmax
                (excluded).
  los           two pairs 1000 Mpc/h from the observer, one radial, one
                transverse, nmu 4: mu bins from each end (radial: 1 and 4
                after clamping; transverse: 2 and 3).
Run: python tests/golden/make_golden.py
"""
import json
import math
import os

HERE = os.path.dirname(os.path.abspath(__file__))


def bin_of(d, rmin, rmax, nbins):
    if d <= rmin or d >= rmax:
        return 0
    return min(int(math.floor((d - rmin) * (1.0 / ((rmax - rmin) / nbins)))) + 1, nbins)


def main():
    cases = []
    # equilateral triangle
    s = 5.0
    pts = [[0.0, 0.0, 0.0], [s, 0.0, 0.0], [s / 2, s * math.sqrt(3.0) / 2, 0.0]]
    cases.append(dict(
        name="equilateral", xyz=pts, w=[1.0, 1.0, 1.0], n_data=3, rmin=1.0, rmax=10.0,
        nbins=3, nmu=1,
        # 2PCF: 6 directed galaxy-galaxy pairs in bin 2
        counts2={"2,1,0": 6},
        # 3PCF: one triangle, rooted at each vertex, configuration (2,2,2) = 7
        counts3={"7,1,0": 3},
        N2_3={"7,1": 3 * (1.0 / 3.0) ** 3}))
    # collinear points on bin edges
    xs = [0.0, 3.0, 4.0, 7.0, 10.0, 11.0]
    pts = [[x, 0.0, 0.0] for x in xs]
    counts2 = {}
    for i, a in enumerate(xs):
        for j, b in enumerate(xs):
            if i == j:
                continue
            bb = bin_of(abs(b - a), 1.0, 10.0, 3)
            if bb:
                k = f"{bb},1,0"
                counts2[k] = counts2.get(k, 0) + 1
    # written out: bin 1 {0-3, 4-7, 7-10}, bin 2 {0-4, 3-7, 4-10, 7-11},
    # bin 3 {0-7, 3-10, 3-11, 4-11}; each pair counted from both ends
    assert counts2 == {"1,1,0": 6, "2,1,0": 8, "3,1,0": 8}, counts2
    cases.append(dict(name="collinear", xyz=pts, w=[1.0] * 6, n_data=6, rmin=1.0, rmax=10.0,
                      nbins=3, nmu=1, counts2=counts2))
    # line of sight: observer at the origin, nmu = 4
    pts = [[1000.0, 0.0, 0.0], [1005.0, 0.0, 0.0], [0.0, 1000.0, 0.0], [0.0, 1000.0, 5.0]]
    # radial pair: theta(0->1) = -1 -> bin 1; theta(1->0) = +1 -> bin 5 -> 4
    # transverse pair: theta = -/+ 12.5/(|m| 5) ~ -/+0.0025 -> bins 2 / 3
    # separation 5 -> radial bin 2 of 3 (rmin 1, rmax 10)
    cases.append(dict(name="los", xyz=pts, w=[1.0] * 4, n_data=4, rmin=1.0, rmax=10.0,
                      nbins=3, nmu=4,
                      counts2={"2,1,0": 1, "2,4,0": 1, "2,2,0": 1, "2,3,0": 1},
                      edges={"0,1": [2, 1], "1,0": [2, 4], "2,3": [2, 2], "3,2": [2, 3]}))
    with open(os.path.join(HERE, "known_answers.json"), "w") as f:
        json.dump(cases, f, indent=1)


if __name__ == "__main__":
    main()
