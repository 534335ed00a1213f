"""Regenerates the committed golden fixtures in this folder.

Run where a checkout of the reference is available, naming its root in
CLE_REFERENCE_ROOT (the directory holding data/ and demo/):

    CLE_REFERENCE_ROOT=/path/to/pyclesperanto_prototype python tests/golden/make_golden.py

Outputs:
  blobs.npz           -- data/blobs.tif of the reference (254x256 uint8), read
                         with PIL; the input of the reference's blob tests and
                         demo notebooks.
  known_answers.json  -- numbers printed in the reference's own test files and
                         demo-notebook outputs for that image, extracted here
                         from the notebook JSON (cell outputs) so that their
                         provenance is explicit.
"""
import json
import os
import re

import numpy as np
from PIL import Image

REF = os.environ.get("CLE_REFERENCE_ROOT")
HERE = os.path.dirname(os.path.abspath(__file__))


def cell_text(nb_path, cell):
    nb = json.load(open(os.path.join(REF, nb_path)))
    outs = nb["cells"][cell].get("outputs", [])
    parts = []
    for o in outs:
        if "text" in o:
            parts.append("".join(o["text"]))
        elif "data" in o and "text/plain" in o["data"]:
            parts.append("".join(o["data"]["text/plain"]))
    return "\n".join(parts)


def corners(text):
    """Parse a numpy summary print 'OCLArray([[a, b, c, ..., d, e, f], ...'
    into its top-right and bottom-right 3x3 corner values."""
    rows = re.findall(r"\[\s*([^\[\]]+?)\]", text)
    vals = []
    for r in rows:
        if "..." not in r:
            continue
        left, right = r.split("...")
        lv = [float(v) for v in left.replace(",", " ").split()]
        rv = [float(v) for v in right.replace(",", " ").split()]
        vals.append((lv, rv))
    return {"top_left": [v[0] for v in vals[:3]], "top_right": [v[1] for v in vals[:3]],
            "bottom_left": [v[0] for v in vals[3:6]], "bottom_right": [v[1] for v in vals[3:6]]}


def main():
    if not REF or not os.path.isdir(os.path.join(REF, "data")):
        raise SystemExit("set CLE_REFERENCE_ROOT to the reference checkout (the directory with data/ and demo/)")
    img = np.asarray(Image.open(os.path.join(REF, "data", "blobs.tif")))
    np.savez_compressed(os.path.join(HERE, "blobs.npz"), blobs=img)

    lab = "demo/segmentation/labeling.ipynb"
    stats = "demo/basics/label_statistics.ipynb"
    ka = {
        "source_image": "data/blobs.tif",
        # tests/test_connected_components_labeling_box.py:34-64
        "blur1_otsu_ccl_num_labels": {"value": 62,
                                      "cite": "tests/test_connected_components_labeling_box.py:64"},
        # demo/segmentation/labeling.ipynb cells 6 and 11: CCL box of raw > 100
        "ccl_box_raw_gt_100": {"corners": corners(cell_text(lab, 6)), "max": 65,
                               "cite": lab + " cells 6, 11"},
        # cells 13-14: gauss_otsu_labeling outline_sigma 1 and 5
        "gauss_otsu_1": {"corners": corners(cell_text(lab, 13)), "cite": lab + " cell 13"},
        "gauss_otsu_5": {"corners": corners(cell_text(lab, 14)), "cite": lab + " cell 14"},
        # cells 19-20: voronoi_otsu_labeling
        "vol_spot1_outline1": {"corners": corners(cell_text(lab, 19)), "cite": lab + " cell 19"},
        "vol_spot3.2_outline1": {"corners": corners(cell_text(lab, 20)), "cite": lab + " cell 20"},
        # label_statistics.ipynb cells 2, 7, 8: voronoi_otsu_labeling(spot_sigma=3.5)
        "vol_spot3.5_outline2": {"corners": corners(cell_text(stats, 2)), "cite": stats + " cell 2"},
    }
    # statistics table rows (labels 1-5 and 61-65): bbox columns, cell 7
    t7 = cell_text(stats, 7)
    rows = {}
    for line in t7.splitlines():
        m = re.match(r"^\s*(\d+)\s+(\d+)\s+(\d+)\s+([\d.]+)\s+([\d.]+)\s+([\d.]+)\s+([\d.]+)\s*\\?$", line)
        if m:
            rows[int(m.group(2))] = {"bbox_min_x": float(m.group(4)), "bbox_min_y": float(m.group(5)),
                                     "bbox_min_z": float(m.group(6)), "bbox_max_x": float(m.group(7))}
    for line in t7.splitlines():
        m = re.match(r"^\s*(\d+)\s+([\d.]+)\s+([\d.]+)\s+([\d.]+)\s+([\d.]+)\s+\.\.\.", line)
        if m:
            idx = int(m.group(1))
            lab_id = idx + 1
            if lab_id in rows:
                rows[lab_id].update({"bbox_max_y": float(m.group(2)), "bbox_max_z": float(m.group(3)),
                                     "bbox_width": float(m.group(4)), "bbox_height": float(m.group(5))})
    ka["vol_spot3.5_outline2"]["num_labels"] = 65
    ka["vol_spot3.5_outline2"]["table_rows"] = rows
    # table.describe(), cell 8: count / mean / min / max of bbox columns
    t8 = cell_text(stats, 8)
    desc = {}
    lines = t8.splitlines()
    header = None
    for line in lines:
        toks = line.split()
        if not toks:
            continue
        if toks[0] in ("count", "mean", "std", "min", "25%", "50%", "75%", "max") and header:
            vals = [t for t in toks[1:] if t not in ("...", "\\")]
            for h, v in zip(header, vals):
                desc.setdefault(h, {})[toks[0]] = float(v)
        elif not re.match(r"^[\d.]", toks[0]):
            header = [t for t in toks if t not in ("...", "\\")]
    ka["vol_spot3.5_outline2"]["describe"] = desc
    ka["vol_spot3.5_outline2"]["cite"] = stats + " cells 2, 7, 8"
    with open(os.path.join(HERE, "known_answers.json"), "w") as f:
        json.dump(ka, f, indent=1, sort_keys=True)
    print("wrote", os.listdir(HERE))


if __name__ == "__main__":
    main()
