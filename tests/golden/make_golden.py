"""Writes tests/golden/golden.npz from the reference's own CPU code.

Run where the reference sources exist and oracle/_ref/gatref has been built (make -C oracle):

    python tests/golden/make_golden.py

Inputs come from the library's seeded generator; the fixture stores the generator parameters,
a SHA-256 of every generated input (so a changed generator fails loudly) and the reference's
outputs: Grid (GT-quadtree) id sets, candidate leaves and layout digest; STIG id sets and layout
digest; FSG layout digest; EDR distances at two eps values; FV lower bounds; top-k distance
multisets; FVTable::findNeighbor and getIdxFromXY tables (edge cells included).
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from gat_b200 import data as D  # noqa: E402
from oracle import pyoracle as po  # noqa: E402

BOX = D.BOX


def digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def inputs():
    """The fixture inputs, regenerated identically by tests/test_golden.py."""
    t = D.walks(D.lengths(4000, 0, 0, 0, 1, 200, 7), 7)
    q = np.concatenate([D.boxes(120, 1, 0.005, 0.12, 8),
                        np.array([[121.0, 30.7, 121.01, 30.71], [121.995, 31.69, 122.05, 31.8], [120.9, 30.6, 121.2, 30.75],
                                  [121.5, 31.2, 121.5, 31.2], [122.5, 32.0, 122.6, 32.1]], np.float32)])
    la = np.array([1, 1, 2, 2, 3, 16, 100, 129, 257, 300] + list(D.lengths(190, 2, 0, 0, 1, 400, 9)), np.int32)
    lb = np.array([1, 5, 2, 7, 3, 16, 100, 128, 256, 300] + list(D.lengths(190, 2, 0, 0, 1, 400, 10)), np.int32)
    a, b = D.pairs(la, lb, 11)
    tk = D.walks(D.lengths(3000, 1, float(np.log(200.0)), 0.6, 32, 1024, 12), 12)
    qids = D.sample_ids(6, tk.n, 13)
    return t, q, la, a, lb, b, tk, qids


def main():
    if not po.ref_available():
        raise SystemExit("oracle/_ref/gatref missing: build it with `make -C oracle` next to the reference sources")
    R = po.RefRunner()
    t, q, la, a, lb, b, tk, qids = inputs()
    out = {"input_digest": np.array(digest(t.lengths, t.lon, t.lat, q, la, a, lb, b, tk.lengths, tk.lon, tk.lat, qids))}
    r = R.gtq(t, q, BOX, 0.01, 64, layout=True)
    out.update(gtq_id_off=r["id_off"], gtq_ids=r["ids"], gtq_cand_off=r["cand_off"], gtq_cand_node=r["cand_node"],
               gtq_cand_level=r["cand_level"], gtq_meta=r["meta"],
               gtq_layout=np.array(digest(r["px"], r["py"], r["ptid"], r["cell_start"], r["cell_end"])),
               gtq_fv=np.array(digest(r["fv_off"], r["fv_cell"], r["fv_count"])))
    r = R.stig(t, q, 256, layout=True)
    out.update(stig_id_off=r["id_off"], stig_ids=r["ids"], stig_blk_off=r["blk_off"], stig_blk=r["blk"],
               stig_layout=np.array(digest(r["px"], r["py"], r["ptid"])))
    r = R.fsg(t, BOX, 0.01)
    out.update(fsg_meta=r["meta"], fsg_layout=np.array(digest(r["px"], r["py"], r["ptid"], r["cell_start"], r["cell_end"])))
    out["edr_5e-4"] = R.edr(la, a, lb, b, 5e-4)["dist"]
    out["edr_5e-3"] = R.edr(la, a, lb, b, 5e-3)["dist"]
    out["fvlb"] = R.fvlb(tk, qids, BOX, 0.0025)
    rt = R.topk(tk, qids, BOX, 0.0025, 16, 5e-4)
    out["topk_dist_sorted"] = np.sort(rt["dist"], axis=1)
    vc = (512 * 512) >> 2
    cells = np.array([0, 1, 2, 3, 5, 170, 255, 256, 1023, 4096, 21845, 43690, 65535, 65534, 32768], np.int32)
    nb, grid = R.nbr(cells, vc)
    out.update(nbr_cells=cells, nbr=nb, idx_grid=grid)
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **out)
    print("wrote", os.path.join(HERE, "golden.npz"), {k: np.asarray(v).shape for k, v in out.items()})


if __name__ == "__main__":
    main()
