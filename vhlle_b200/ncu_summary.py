"""Summaries of Nsight Compute CSV captures of the step kernels, in the form
bench.py reads (profiles/traffic.json, profiles/fp64.json) and as a text
table of the launch list.

    python -m vhlle_b200.ncu_summary traffic CSV GRID OUT.json   # dram bytes per launch
    python -m vhlle_b200.ncu_summary fp64 CSV GRID OUT.json      # FP64 operations per launch
    python -m vhlle_b200.ncu_summary launches CSV                # per kernel: launches, time, share

CSV is ncu's `--csv --log-file` output of a capture of bench.py's timed
region (`--nvtx --nvtx-include timed/`); GRID is the workload's nx,ny,nz.
Launches are grouped under the kernel names bench.py's per-kernel profile
uses (k_face_x/y/z by direction, k_relax_list counted with k_is_relax, the
freeze-out kernels as "surface"), each kind's values in launch order.
"""
from __future__ import annotations

import collections
import csv
import io
import json
import re
import sys

FP64_METRICS = ("sm__sass_thread_inst_executed_op_dadd_pred_on.sum",
                "sm__sass_thread_inst_executed_op_dmul_pred_on.sum",
                "sm__sass_thread_inst_executed_op_dfma_pred_on.sum")
DRAM_METRICS = ("dram__bytes_read.sum", "dram__bytes_write.sum")
SURFACE = ("k_surf_", "k_scan_excl", "k_sum_cols", "k_corona")


def kind_of(name: str) -> str:
    """bench.py's kernel kind of an ncu kernel name."""
    base = re.sub(r"^void\s+", "", name).split("(")[0]
    base = base.replace("vh::", "")
    short = base.split("<")[0]
    if short == "k_face":
        d = re.search(r"<\s*(\d)", base)
        return "k_face_" + {"1": "x", "2": "y", "3": "z"}.get(d.group(1) if d else "", "?")
    if short == "k_relax_list":
        return "k_is_relax"
    if any(short.startswith(p) for p in SURFACE):
        return "surface"
    return short


def read_rows(path: str):
    """[(launch id, kind, {metric: value})] in launch order."""
    txt = open(path).read()
    start = txt.index('"ID"')
    rows = list(csv.reader(io.StringIO(txt[start:])))
    hdr = rows[0]
    col = {h: i for i, h in enumerate(hdr)}
    launches = collections.OrderedDict()
    for r in rows[1:]:
        if len(r) < len(hdr):
            continue
        lid = int(r[col["ID"]])
        name = r[col["Kernel Name"]]
        ent = launches.setdefault(lid, (kind_of(name), {}))
        v = r[col["Metric Value"]].replace(",", "")
        try:
            ent[1][r[col["Metric Name"]]] = float(v)
        except ValueError:
            pass
    return [(lid, k, m) for lid, (k, m) in launches.items()]


def per_launch(rows, value, merge=("k_is_relax",)):
    """{kind: [value per launch]}; for the kinds in `merge`, consecutive
    launches of that kind with no other kernel between them (k_relax_list
    then k_is_relax) count as one launch."""
    out = collections.OrderedDict()
    prev = None
    for _, k, m in rows:
        v = value(m)
        if k in merge and prev == k and out[k]:
            out[k][-1] += v
        else:
            out.setdefault(k, []).append(v)
        prev = k
    return out


def fp64_flops(m) -> float:
    return (m.get(FP64_METRICS[0], 0.0) + m.get(FP64_METRICS[1], 0.0) +
            2.0 * m.get(FP64_METRICS[2], 0.0))


def dram_bytes(m) -> float:
    return m.get(DRAM_METRICS[0], 0.0) + m.get(DRAM_METRICS[1], 0.0)


def write_json(path: str, grid: str, key: str, data, source: str) -> None:
    try:
        doc = json.load(open(path))
    except (OSError, ValueError):
        doc = {}
    doc.setdefault("_source", {})[grid] = source
    doc[grid] = {k: {key: v} for k, v in data.items()}
    with open(path, "w") as f:
        json.dump(doc, f, indent=1)
        f.write("\n")


def launch_table(rows) -> str:
    t = collections.OrderedDict()
    for _, k, m in rows:
        n, s = t.get(k, (0, 0.0))
        t[k] = (n + 1, s + m.get("gpu__time_duration.sum", 0.0))
    total = sum(s for _, s in t.values()) or 1.0
    lines = ["| kernel | launches | total ms | share |", "|---|---|---|---|"]
    for k, (n, s) in sorted(t.items(), key=lambda kv: -kv[1][1]):
        lines.append("| %s | %d | %.3f | %.3f |" % (k, n, s / 1e6, s / total))
    return "\n".join(lines)


def main(argv):
    if len(argv) >= 4 and argv[0] in ("traffic", "fp64"):
        rows = read_rows(argv[1])
        if argv[0] == "traffic":
            data = per_launch(rows, dram_bytes)
            write_json(argv[3], argv[2], "bytes_per_launch", data,
                       "ncu --metrics " + ",".join(DRAM_METRICS))
        else:
            data = per_launch(rows, fp64_flops)
            write_json(argv[3], argv[2], "flops_per_launch", data,
                       "ncu --metrics " + ",".join(FP64_METRICS) + " (flops = add + mul + 2 fma)")
        return 0
    if len(argv) == 2 and argv[0] == "launches":
        print(launch_table(read_rows(argv[1])))
        return 0
    sys.stderr.write(__doc__)
    return 2


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
