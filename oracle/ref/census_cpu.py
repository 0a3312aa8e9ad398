"""Census of the reference's CPU correction on seeded 2-D fields.

Runs oracle/_ref/ref_cpu and oracle/_ref/ref_cpu_zero (built by
build_ref_cpu.sh from src/ExtreM.cpp + main.cpp) on fields of the synthetic
generator and reports, per field, whether the program writes its corrected
field or dies, next to the number of maxima the CPU classification finds.

The CPU classification (classifyVertex1, src/ExtreM.cpp:703-891) takes the star
of a vertex from the 6-direction adjacency (computeAdjacency :545-573, in 2-D
the four axis neighbours E, W, N, S) and joins star vertices only along the
edges of the triangles that hold the vertex (get_vertex_traingle :1584-1594,
getVerticesFromTriangleID1 :597-629).  The only such edges between axis
neighbours are E-N and W-S, so an interior vertex whose four neighbours are
all lower has two lower components and is typed 1, not 4 (and an interior
minimum is typed 2).  Maxima (type 4) and minima (type 0) occur only at the
corners (0,0) and (W-1,H-1).  The CP lists then hold at most two extrema,
findAscPaths / findDesPaths read computeCP's tempArray at every manifold root
(:1617, :1660), written only at listed extrema (:2004-2012), and
computelargestSaddlesForMax / computesmallestSaddlesForMin (:2312-2368,
main.cpp:111-112) index `maximum[...]` / `minimum[...]` with what they read:
an empty list faults at once, other garbage later.

Test infrastructure only:  python -m oracle.ref.census_cpu [--quick]
"""

import argparse
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(HERE, "..", "_ref")


def cpu_types(f):
    """The CPU classification of a 2-D field (H, W), x fastest.

    Lower/upper by (value, id); components counted with the E-N and W-S link
    edges; the codes of classifyVertex1 (:884-891).
    """
    h, w = f.shape
    ids = np.arange(h * w).reshape(h, w)
    out = np.empty((h, w), np.int8)
    for y in range(h):
        for x in range(w):
            v, i = f[y, x], ids[y, x]
            nb = {}
            for name, (dx, dy) in (("E", (1, 0)), ("W", (-1, 0)), ("N", (0, 1)), ("S", (0, -1))):
                xx, yy = x + dx, y + dy
                if 0 <= xx < w and 0 <= yy < h:
                    u, j = f[yy, xx], ids[yy, xx]
                    nb[name] = u < v or (u == v and j < i)
            lo = [k for k, low in nb.items() if low]
            up = [k for k, low in nb.items() if not low]

            def comps(s):
                c = len(s)
                c -= ("E" in s and "N" in s)
                c -= ("W" in s and "S" in s)
                return c
            lc, uc = comps(lo), comps(up)
            if lc == 0 and uc == 1:
                t = 0
            elif lc == 1 and uc == 0:
                t = 4
            elif lc == 1 and uc == 1:
                t = 5
            elif lc > 1 and uc > 1:
                t = 3
            elif lc > 1:
                t = 1
            elif uc > 1:
                t = 2
            else:
                t = 5
            out[y, x] = t
    return out


def run(binary, d, w, h, er, threads):
    env = dict(os.environ, EXTREMZ_REF_DECP=os.path.join(d, "decp.bin"))
    if threads:
        env["OMP_THREAD_LIMIT"] = str(threads)
    fixed = os.path.join(d, "fixed.bin")
    if os.path.exists(fixed):
        os.remove(fixed)
    try:
        p = subprocess.run([binary, f"{os.path.join(d, 'orig.bin')},{w},{h},1", str(er), "x"],
                           cwd=d, env=env, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                           timeout=60)
    except subprocess.TimeoutExpired:
        return "no end in 60 s", None
    ok = os.path.exists(fixed)
    if ok:
        return "ok", np.fromfile(fixed, "<f8")
    return ("SIGSEGV" if p.returncode == -11 else f"rc {p.returncode}"), None


def main():
    sys.path.insert(0, os.path.join(HERE, "..", ".."))
    from extrem_z_b200 import synth
    ap = argparse.ArgumentParser()
    ap.add_argument("--quick", action="store_true")
    a = ap.parse_args()
    for b in ("ref_cpu", "ref_cpu_zero"):
        if not os.path.exists(os.path.join(REF, b)):
            sys.exit(f"{b} missing: run oracle/ref/build_ref_cpu.sh")
    seeds = range(1, 4) if a.quick else range(1, 13)
    sizes = [(48, 40), (64, 64), (96, 80), (128, 128)]
    er = 1e-3
    print("| field | maxima (CPU types) | stock, 1 thread | stock, default threads | "
          "zero-filled, 1 thread | zero-filled, default threads |")
    print("|---|---|---|---|---|---|")
    tally = [0, 0, 0, 0]
    total = 0
    for s in seeds:
        for (w, h) in sizes:
            fld = synth.make_field(w, h, 1, n_gauss=16, seed=s, rel=er, dtype=np.float64)
            with tempfile.TemporaryDirectory() as d:
                fld.f.astype("<f8").tofile(os.path.join(d, "orig.bin"))
                fld.decp.astype("<f8").tofile(os.path.join(d, "decp.bin"))
                t = cpu_types(fld.f.reshape(h, w))
                maxima = [int(i) for i in np.flatnonzero(t.ravel() == 4)]
                res = []
                outs = []
                for k, (b, th) in enumerate((("ref_cpu", 1), ("ref_cpu", 0),
                                             ("ref_cpu_zero", 1), ("ref_cpu_zero", 0))):
                    r, o = run(os.path.join(REF, b), d, w, h, er, th)
                    res.append(r)
                    outs.append(o)
                    tally[k] += r == "ok"
                if outs[2] is not None and outs[3] is not None:
                    res[3] += " (same)" if np.array_equal(outs[2], outs[3]) else " (differs)"
            total += 1
            print(f"| {w}x{h} seed {s} | {maxima} | " + " | ".join(res) + " |")
    print(f"\ncompleted: stock 1 thread {tally[0]}/{total}, stock {tally[1]}/{total}, "
          f"zero-filled 1 thread {tally[2]}/{total}, zero-filled {tally[3]}/{total}")


if __name__ == "__main__":
    main()
