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
                (excluded); in log bins (rmin 1, rmax 100, 2 bins) a
                separation on the edge at 10.
  los           two pairs 1000 Mpc/h from the observer, one radial, one
                transverse, nmu 4: mu bins from each end (radial: 1 and 4
                after clamping; transverse: 2 and 3).
  los_triangle  equilateral triangle of side 5 across the line of sight,
                nmu 4: edge mu bins 2 / 3, every root's find_normal bin 4.
  tetrahedron   regular tetrahedron of edge sqrt(32) (radial bin 2) and its
                centre, sqrt(12) from every vertex (bin 1); rmin 1, rmax 10,
                3 bins.  Vertices 0-2 are galaxies, vertex 3 and the centre
                (id 4) randoms, unit weights.  2PCF, 3PCF and 4PCF answers
                below are derived by hand from the reference loops; the 4PCF
                pins the perimeter order, the root-row length rule (every row
                holds 4 > 3 neighbours), the non-canonical table entries
                (taken as 0) and the six disconnected-term gates; the
                -equi and -tetra answers likewise, the closed-form
                weight gradients of the 2/3/4PCF sums, and the counts with
                the centre as a buffer point.
Run: python tests/golden/make_golden.py
"""
import itertools
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
    # the same points in log bins: rmin 1, rmax 100, 2 bins, edges 1, 10, 100
    # (gramsci.F90:136-139, :334-335).  Separations 3, 4, 7 (three pairs
    # each), 6 and 8 fall in bin 1; 10 lands exactly on the edge
    # (log10(10) = 1, t = 1.0) and 11 above it: bin 2; the two pairs at
    # d = 1 = rmin are excluded
    log2 = {}
    for i, a in enumerate(xs):
        for j, b in enumerate(xs):
            d = abs(b - a)
            if i == j or d <= 1.0 or d >= 100.0:
                continue
            bb = min(int(math.floor((math.log10(d) - math.log10(1.0)) * (1.0 / (2.0 / 2)))) + 1, 2)
            k = f"{bb},1,0"
            log2[k] = log2.get(k, 0) + 1
    assert log2 == {"1,1,0": 22, "2,1,0": 4}, log2
    cases.append(dict(name="collinear", xyz=pts, w=[1.0] * 6, n_data=6, rmin=1.0, rmax=10.0,
                      nbins=3, nmu=1, counts2=counts2,
                      log_case=dict(rmin=1.0, rmax=100.0, nbins=2, counts2=log2,
                                    edges={"0,4": [2, 1], "4,0": [2, 1], "0,5": [2, 1],
                                           "0,3": [1, 1]})))
    # line of sight: observer at the origin, nmu = 4
    pts = [[1000.0, 0.0, 0.0], [1005.0, 0.0, 0.0], [0.0, 1000.0, 0.0], [0.0, 1000.0, 5.0]]
    # radial pair: theta(0->1) = -1 -> bin 1; theta(1->0) = +1 -> bin 5 -> 4
    # transverse pair: theta = -/+ 12.5/(|m| 5) ~ -/+0.0025 -> bins 2 / 3
    # separation 5 -> radial bin 2 of 3 (rmin 1, rmax 10)
    cases.append(dict(name="los", xyz=pts, w=[1.0] * 4, n_data=4, rmin=1.0, rmax=10.0,
                      nbins=3, nmu=4,
                      counts2={"2,1,0": 1, "2,4,0": 1, "2,2,0": 1, "2,3,0": 1},
                      edges={"0,1": [2, 1], "1,0": [2, 4], "2,3": [2, 2], "3,2": [2, 3]}))
    # equilateral triangle of side 5 across the line of sight, 1000 Mpc/h
    # out, nmu 4.  m.s = (|p_i|^2 - |p_j|^2) / 2 is -62.5, -37.5, 25 for the
    # pairs (0,1), (0,2), (1,2): cosines -0.0125, -0.0075, 0.005 seen from
    # the first vertex, so mu bin 2 from one end and 3 from the other
    # (floor((theta + 1) * 2) + 1).  The roots' mu pairs are (2,2), (3,3),
    # (3,2); find_normal (gramsci.F90:1611-1625) maps bin centres -0.25 /
    # 0.25 through 1.1547 * sqrt(0.6875) * 4 = 3.83 and
    # 1.1547 * sqrt(0.5625) * 4 = 3.46 to bin 4 for all three.
    h = 2.5 * math.sqrt(3.0)
    pts = [[10.0, 0.0, 1000.0], [15.0, 0.0, 1000.0], [12.5, h, 1000.0]]
    cases.append(dict(
        name="los_triangle", xyz=pts, w=[1.0] * 3, n_data=3, rmin=1.0, rmax=10.0,
        nbins=3, nmu=4,
        counts2={"2,2,0": 3, "2,3,0": 3},
        counts3={"7,4,0": 3},
        N2_3={"7,4": 3 * (1.0 / 3.0) ** 3},
        edges={"0,1": [2, 2], "1,0": [2, 3], "0,2": [2, 2], "2,0": [2, 3], "1,2": [2, 3],
               "2,1": [2, 2]}))
    # regular tetrahedron + centre.  Every separation is sqrt(32) (vertex to
    # vertex, t = (5.657 - 1)/3 = 1.55, bin 2) or sqrt(12) (to the centre,
    # t = 0.82, bin 1), far from the bin edges 1, 4, 7, 10.
    pts = [[102.0, 102.0, 102.0], [102.0, 98.0, 98.0], [98.0, 102.0, 98.0],
           [98.0, 98.0, 102.0], [100.0, 100.0, 100.0]]
    for i in range(4):
        for j in range(i + 1, 4):
            assert sum((a - b) ** 2 for a, b in zip(pts[i], pts[j])) == 32.0
        assert sum((a - b) ** 2 for a, b in zip(pts[i], pts[4])) == 12.0
    g, r = 1.0 / 3.0, -1.0 / 2.0  # normalised weights: 3 galaxies, 2 randoms
    nc4 = 0  # rank of (2,2,2,2) among i<=j<=k<=l<=3, lexicographic
    for t in sorted(q for q in itertools.product(range(1, 4), repeat=4) if list(q) == sorted(q)):
        nc4 += 1
        if t == (2, 2, 2, 2):
            break
    assert nc4 == 11
    cases.append(dict(
        name="tetrahedron", xyz=pts, w=[1.0] * 5, n_data=3, rmin=1.0, rmax=10.0,
        nbins=3, nmu=1, rtol=1e-13,
        # directed pairs, category 2*random(root) + random(neighbour):
        # vertex-vertex (bin 2): galaxy-galaxy 6, galaxy->v3 3, v3->galaxy 3;
        # centre (bin 1): galaxy->centre 3, centre->galaxy 3, v3<->centre 2
        counts2={"2,1,0": 6, "2,1,1": 3, "2,1,2": 3, "1,1,1": 3, "1,1,2": 3, "1,1,3": 2},
        # 3PCF, each triangle once per vertex: the four faces are (2,2,2) =
        # rank 7, face 012 with no random, the three faces with v3 with one;
        # the six centre triangles are (1,1,2) = rank 2, one random (the
        # centre) for galaxy pairs, two for pairs with v3
        counts3={"7,1,0": 3, "7,1,1": 9, "2,1,1": 9, "2,1,2": 9},
        N2_3={"7,1": 3 * g ** 3 + 9 * g * g * r, "2,1": 9 * g * g * r + 9 * g * r * r},
        # 4PCF: a vertex root's triples with the centre (always the largest
        # id) have the perimeter (2,2,1,1), the centre root's (1,2,2,1):
        # both non-canonical, so only the tetrahedron contributes, once
        # from each vertex, at (cfg 11, bin(i,b) 2, bin(a,c) 2) with one
        # random (v3)
        counts4={"11,2,2,1": 4},
        N2_4={"11,2,2": 4 * g ** 3 * r},
        # disconnected terms: roots 0-2 see v3 as their last member c (gate
        # of terms 1 and 2, pairs (i,a) and (i,b)); root 3 is the random
        # gate of terms 4-6 (pairs among its three galaxy members); all
        # pairs are galaxy pairs, so discR is 0
        dcount4={"11,2,2,1,0": 3, "11,2,2,2,0": 3, "11,2,2,4,0": 1, "11,2,2,5,0": 1,
                 "11,2,2,6,0": 1},
        discN4={"11,2,2,1": 3 * g * g, "11,2,2,2": 3 * g * g, "11,2,2,4": g * g,
                "11,2,2,5": g * g, "11,2,2,6": g * g},
        # -equi (gramsci.F90:402-446): triangles with three edges in one bin
        # are the four faces (bin 2), rooted at each vertex
        counts_equi={"2,1,0": 3, "2,1,1": 9},
        N2_equi={"2,1": 3 * g ** 3 + 9 * g * g * r},
        # -tetra (:548-640): cliques with six edges in one bin, no row-length
        # rule: the tetrahedron from each vertex.  Its disconnected terms
        # are triple products with the gate vertex's weight: roots 0-2 have
        # v3 as id3 (gate of terms 1 and 2), root 3 is the random root (gate
        # of terms 4, 5, 6); term 3's gate id1 is always a galaxy
        counts_tetra={"2,1": 4},
        N2_tetra={"2": 4 * g ** 3 * r},
        discN_tetra={"2,1": 3 * r * g * g, "2,2": 3 * r * g * g, "2,4": r * g * g,
                     "2,5": r * g * g, "2,6": r * g * g},
        edges={"0,1": [2, 1], "0,4": [1, 1], "4,3": [1, 1]},
        # weight gradients of L = sum(N2) (every cotangent 1), normalised
        # weights w = (g, g, g, r, r).  All ten pairs are edges and the ten
        # triples triangles: 2PCF dL/dw_k = 2 (sum(w) - w_k) = -2 w_k since
        # sum(w) = 0; 3PCF (each triangle rooted 3 times) dL/dw_k = 3 e2 of
        # the other four weights; 4PCF (the tetrahedron rooted 4 times)
        # dL/dw_k = 4 * product of the other three vertices, 0 for the centre
        grad2=[-2 * g] * 3 + [-2 * r] * 2,
        grad3=[3 * (g * g + 4 * g * r + r * r)] * 3 + [3 * (3 * g * g + 3 * g * r)] * 2,
        grad4=[4 * g * g * r] * 3 + [4 * g ** 3, 0.0],
        # the centre as a buffer point (gramsci.F90:363,476,672): it roots
        # nothing, so its 3 + 1 directed pairs go and the six centre
        # triangles are counted from two vertices instead of three; the
        # 4PCF is unchanged because a buffer point still counts in its
        # neighbours' rows (every vertex row keeps 4 > 3 entries)
        buffer_case=dict(
            buffer=[0, 0, 0, 0, 1],
            counts2={"2,1,0": 6, "2,1,1": 3, "2,1,2": 3, "1,1,1": 3, "1,1,3": 1},
            counts3={"7,1,0": 3, "7,1,1": 9, "2,1,1": 6, "2,1,2": 6},
            N2_3={"7,1": 3 * g ** 3 + 9 * g * g * r, "2,1": 6 * g * g * r + 6 * g * r * r})))
    with open(os.path.join(HERE, "known_answers.json"), "w") as f:
        json.dump(cases, f, indent=1)


if __name__ == "__main__":
    main()
