"""Extract reference-printed values from the reference's own sample logs into a fixture.

Run here (where the reference tree exists): ``python tests/golden/extract_reference_logs.py``.
It reads the O2 sample runs of RSDFT (cubic cell, AX = 18.89726878 bohr, 48^3 grid, Md = 6)
under samples_for_supercomputers/*/02_O2-molecule_optimize/real8/result/a.log and the Si band
runs (*/01_Si_band/result/a.log) and writes reference_logs.json beside this script: the cell,
the grid and the init_kinetic table the reference printed (lap(m), coef_lap(1:3, m), nab(m),
coef_nab(1:3, m), ggg), and generate_bz's k-point list (MMM divisions, kbb, weight_bz).  The tests use the
JSON file only, so they run where the reference tree is absent.
"""
import glob
import json
import os
import re

REF = "/root/reference/samples_for_supercomputers"
HERE = os.path.dirname(os.path.abspath(__file__))


def parse(path):
    txt = open(path).read().splitlines()
    out = {"source": os.path.relpath(path, os.path.dirname(REF))}
    for i, line in enumerate(txt):
        m = re.match(r"\s*AX :\s*([0-9.Ee+-]+)", line)
        if m:
            out["ax"] = float(m.group(1))
        m = re.match(r"\s*Ngrid\(1:3\)=\s*(\d+)\s+(\d+)\s+(\d+)", line)
        if m:
            out["ngrid"] = [int(m.group(k)) for k in (1, 2, 3)]
        if line.strip().startswith("ggg="):
            out["ggg"] = [float(x) for x in line.split("=")[1].split()]
        if re.match(r"\s+lap\s+coef_lap", line):
            rows = []
            for j in range(i + 1, i + 20):
                f = txt[j].split()
                if not f or not re.match(r"^\d+$", f[0]):
                    break
                rows.append([int(f[0])] + [float(x) for x in f[1:]])
            out["lap_table"] = rows
        if re.match(r"\s+nab\s+coef_nab", line):
            rows = []
            for j in range(i + 1, i + 20):
                f = txt[j].split()
                if not f or not re.match(r"^\d+$", f[0]):
                    break
                rows.append([int(f[0])] + [float(x) for x in f[1:]])
            out["nab_table"] = rows
    return out


def parse_bz(path):
    """generate_bz's printed k-point list: the MP divisions and (kbb(1:3), weight_bz) per point."""
    txt = open(path).read().splitlines()
    out = {"source": os.path.relpath(path, os.path.dirname(REF))}
    for i, line in enumerate(txt):
        m = re.match(r"\s*mmm1=\s*(\d+)\s+(\d+)\s+(\d+)", line)
        if m and "mmm" not in out:
            out["mmm"] = [int(m.group(k)) for k in (1, 2, 3)]
        if "kbb   weight_bz" in line and "kpoints" not in out:
            pts = []
            for j in range(i + 1, len(txt)):
                f = txt[j].split()
                if len(f) != 5 or not f[0].isdigit():
                    break
                pts.append([float(x) for x in f[1:]])
            out["kpoints"] = pts
    return out


def main():
    logs = sorted(glob.glob(os.path.join(REF, "*", "02_O2-molecule_optimize", "real8", "result", "a.log")))
    data = [parse(p) for p in logs]
    data = [d for d in data if "lap_table" in d and "ax" in d]
    bz = [parse_bz(p) for p in sorted(glob.glob(os.path.join(REF, "*", "01_Si_band", "result", "a.log")))]
    bz = [b for b in bz if "mmm" in b and b.get("kpoints")]
    json.dump({"kinetic": data, "bz": bz}, open(os.path.join(HERE, "reference_logs.json"), "w"), indent=1)
    print(f"{len(data)} kinetic tables, {len(bz)} k-point lists -> reference_logs.json")


if __name__ == "__main__":
    main()
