"""Extract reference-printed values from the reference's own sample logs into a fixture.

Run here (where the reference tree exists): ``python tests/golden/extract_reference_logs.py``.
It reads the O2 sample runs of RSDFT (cubic cell, AX = 18.89726878 bohr, 48^3 grid, Md = 6)
under samples_for_supercomputers/*/02_O2-molecule_optimize/real8/result/a.log and the Si band
runs (*/01_Si_band/result/a.log) and writes reference_logs.json beside this script: the cell,
the grid and the init_kinetic table the reference printed (lap(m), coef_lap(1:3, m), nab(m),
coef_nab(1:3, m), ggg), and generate_bz's k-point list (MMM divisions, kbb, weight_bz).  From
every O2 log (real8 and complex16 builds) it also takes what read_PSV printed for the oxygen
pseudopotential, the G sphere of Init_Ggrid (Ecut, Gcut, NGgrid, NMGL), construct_ps_initrho's
density sums, the band energies of scf_iter 1 (both spins: they belong to the operator built
from the initial density, the same one the preceding sweeps converged), and what scf_iter 1
prints about the density of those bands (charges, sum |rho_up - rho_down| dV, and the squared
changes of V_loc and rho from the initial ones); and the first SCF cycle's converged state (the
energy terms printed after its SCF END, its last eigenvalues and spin-density sum).  From the Si
band runs (FCC cell, 12^3 grid, 63 k-points) it takes the same set-up prints, the Ewald energy,
the scf_iter 1 eigenvalues of every k-point, the converged SCF energies and last eigenvalues,
and the band energies along the k trajectory (band_eigv).  The tests use the JSON file only, so
they run where the reference tree is absent.
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


def parse_o2(path):
    """O2 set-up prints and the scf_iter 1 eigenvalue table of one log."""
    txt = open(path).read().splitlines()
    out = {"source": os.path.relpath(path, os.path.dirname(REF))}
    psv = {}
    num = r"[-+0-9.Ee]+"
    for i, line in enumerate(txt):
        m = re.match(r"\s*Ecut,Gcut=\s*(%s)\s+(%s)" % (num, num), line)
        if m:
            out["ecut"], out["gcut"] = float(m.group(1)), float(m.group(2))
        m = re.match(r"\s*NGgrid=\s*(\d+)", line)
        if m:
            out["nggrid"] = int(m.group(1))
        m = re.match(r"\s*NMGL=\s*(\d+)", line)
        if m:
            out["nmgl"] = int(m.group(1))
        if "*** PSV format ***" in line and not psv:
            for j in range(i + 1, i + 40):
                key, _, val = txt[j].partition("=")
                key = key.strip()
                vals = val.split()
                if key == "zatom":
                    psv["zatom"] = float(vals[0])
                elif key == "# of radial mesh points":
                    psv["mr"] = int(vals[0])
                elif key.startswith("r(1)"):
                    psv["r_end"] = float(vals[1])
                elif key == "NRps":
                    psv["nrps"] = [int(v) for v in vals]
                elif key == "# of orbitals":
                    psv["norb"] = int(vals[0])
                elif key == "angular momentum":
                    psv["lo"] = [int(v) for v in vals]
                elif key == "cut off radius":
                    psv["rps"] = [float(v) for v in vals]
                elif key == "Zps":
                    psv["zps"] = float(vals[0])
                elif key == "xc_pot":
                    psv["xc_pot"] = vals[0]
                elif key == "a1,a2,a3,a4":
                    psv["parloc"] = [float(v) for v in vals] + [float(v) for v in txt[j + 1].split()]
                elif key == "Reference":
                    psv["nrf"] = [int(v) for v in vals]
                elif key == "anorm":
                    psv["anorm"] = [float(v) for v in vals]
                elif key == "inorm":
                    psv["inorm"] = [float(v) for v in vals]
                elif key == "sum(cdd)":
                    psv["sum_cdd"] = float(vals[0])
                elif key == "sum(cdc)":
                    psv["sum_cdc"] = float(vals[0])
                    break
            out["psv"] = psv
        if "construct_ps_initrho(start)" in line:
            rows = []
            for j in range(i + 1, i + 20):
                if "construct_ps_initrho(end)" in txt[j]:
                    break
                f = txt[j].split()
                if len(f) == 4 and all(re.match(r"^%s$" % num, x) for x in f):
                    rows.append([float(x) for x in f])
            out["initrho"] = rows
        if re.match(r"-+\s*scf_iter=\s*1$", line) and "esp_scf1" not in out:
            for j in range(i + 1, i + 40):
                t = txt[j].strip()
                if "scf_iter=" in t:
                    break
                if t.startswith("Charge:"):
                    out["charge_scf1"] = [float(x) for x in t.split(":")[1].split()]
                elif t.startswith("sum|rho_up-rho_down|"):
                    out["sum_abs_spin_scf1"] = float(t.split(":")[1])
                elif t.startswith("|Vloc-Vloc0|^2/tol"):
                    out["sqerr_v_scf1"] = [float(x) for x in t.split("=")[1].split("/")[0].split()]
                elif t.startswith("|rho -rho0 |^2/tol"):
                    out["sqerr_rho_scf1"] = [float(x) for x in t.split("=")[1].split("/")[0].split()]
            for j in range(i + 1, i + 40):
                if "esp(n,k,s)" in txt[j]:
                    rows = []
                    for jj in range(j + 1, j + 40):
                        f = txt[jj].split()
                        if len(f) != 8:
                            break
                        rows.append([int(f[0]), int(f[1])] + [float(x) for x in f[2:]])
                    out["esp_scf1"] = rows
                    break
    return out


ENERGY_KEYS = {
    "Total Energy": "total", "Ion-Ion": "ewald", "Local Potential": "local",
    "Ion Local Potential": "ion_local", "Ion Nonlocal Potential": "nonlocal", "Kinetic Energy": "kinetic",
    "Hartree Energy": "hartree", "Exchange-Correlation Energy": "xc", "Exchange Energy": "exchange",
    "Correlation Energy": "correlation", "Sum of eigenvalues": "sum_eigen", "Fermi energy": "fermi",
    "Entropy": "entropy", "Free Energy": "free", "Harris Energy": "harris",
}


def parse_o2_scf(path):
    """The first SCF cycle's converged state (before the atoms move): the energy block printed
    after its SCF END, and the eigenvalue table and sum |rho_up - rho_down| of its last
    iteration."""
    txt = open(path).read().splitlines()
    end = next(i for i, l in enumerate(txt) if "SCF END" in l)
    out = {"source": os.path.relpath(path, os.path.dirname(REF))}
    m = re.search(r"total # of iteration =\s*(\d+)", "\n".join(txt[end:end + 3]))
    out["iterations"] = int(m.group(1)) if m else None
    ene = {}
    start = next(i for i in range(end, len(txt)) if txt[i].strip().endswith("total energy"))
    for line in txt[start + 1:start + 40]:
        if line.startswith("----"):
            break
        for label, key in ENERGY_KEYS.items():
            mm = re.match(re.escape(label) + r"\s+([-+0-9.Ee]+)", line.strip())
            if mm and key not in ene:
                ene[key] = float(mm.group(1))
                break
    out["energies"] = ene
    last = max(i for i in range(end) if "scf_iter=" in txt[i])
    for j in range(last, end):
        t = txt[j].strip()
        if t.startswith("sum|rho_up-rho_down|"):
            out["sum_abs_spin"] = float(t.split(":")[1])
        if "esp(n,k,s)" in t:
            rows = []
            for jj in range(j + 1, j + 40):
                f = txt[jj].split()
                if len(f) != 8:
                    break
                rows.append([int(f[0]), int(f[1])] + [float(x) for x in f[2:]])
            out["esp"] = rows
    return out


def _esp_rows(txt, j, ncol):
    """The eigenvalue table that starts after line j: rows (k, n, values...) of ncol fields."""
    rows = []
    for jj in range(j + 1, len(txt)):
        f = txt[jj].split()
        if len(f) != ncol or not f[0].isdigit():
            break
        rows.append([int(f[0]), int(f[1])] + [float(x) for x in f[2:]])
    return rows


def parse_band_eigv(path):
    """band_eigv of the band-structure run: per trajectory k-point (in trajectory order; the file
    lists them grouped by process) its reduced k and the band energies (mb bands)."""
    txt = open(path).read().splitlines()
    blocks = []
    i = 0
    while i < len(txt):
        f = txt[i].split()
        if len(f) == 6 and f[0].isdigit() and f[1].isdigit() and f[5].isdigit():
            nb = int(f[1])
            blocks.append((int(f[0]), [float(x) for x in f[2:5]],
                           [float(txt[i + 1 + n].split()[1]) for n in range(nb)]))
            i += nb + 1
        else:
            i += 1
    blocks.sort(key=lambda b: b[0])
    return {"source": os.path.relpath(path, os.path.dirname(REF)), "index": [b[0] for b in blocks],
            "kpoints": [b[1] for b in blocks], "esp": [b[2] for b in blocks]}


def parse_si(path):
    """The Si sample's prints (FCC cell, 63 k-points, one spin): the set-up items parse_o2 reads,
    the Ewald energy, the scf_iter 1 eigenvalue table of every k-point (bands 1-9 as printed),
    the converged energy block and iteration count, the last SCF iteration's table, the
    squared changes of V_loc and rho printed at every SCF iteration, and the band run's k
    trajectory (reduced k and the Cartesian step bb dak per point)."""
    txt = open(path).read().splitlines()
    out = {k: v for k, v in parse_o2(path).items() if k != "esp_scf1"}
    out.update({k: v for k, v in parse(path).items() if k != "source"})
    for line in txt:
        m = re.match(r"\s*Eewald\(SYSTYPE=0\)=\s*([-+0-9.Ee]+)", line)
        if m:
            out["ewald"] = float(m.group(1))
            break
    i1 = next(i for i, l in enumerate(txt) if re.match(r"-+\s*scf_iter=\s*1$", l))
    j = next(j for j in range(i1, len(txt)) if "esp(n,k,s)" in txt[j])
    out["esp_scf1"] = _esp_rows(txt, j, 5)
    scf = parse_o2_scf(path)
    out["iterations"] = scf["iterations"]
    out["energies"] = scf["energies"]
    end = next(i for i, l in enumerate(txt) if "SCF END" in l)
    last = max(i for i in range(end) if "scf_iter=" in txt[i])
    j = next(j for j in range(last, end) if "esp(n,k,s)" in txt[j])
    out["esp_last"] = _esp_rows(txt, j, 5)
    i0 = next(i for i, l in enumerate(txt) if l.strip().startswith("nktrj="))
    out["ktrj"] = [[float(x) for x in txt[i].split()[1:7]] for i in range(i0 + 1, i0 + 1 + int(txt[i0].split("=")[1]))]
    out["sqerr_v"] = [float(l.split("=")[1].split("/")[0]) for l in txt[:end] if l.strip().startswith("|Vloc-Vloc0|^2/tol")]
    out["sqerr_rho"] = [float(l.split("=")[1].split("/")[0]) for l in txt[:end] if l.strip().startswith("|rho -rho0 |^2/tol")]
    return out


def main():
    logs = sorted(glob.glob(os.path.join(REF, "*", "02_O2-molecule_optimize", "real8", "result", "a.log")))
    data = [parse(p) for p in logs]
    data = [d for d in data if "lap_table" in d and "ax" in d]
    bz = [parse_bz(p) for p in sorted(glob.glob(os.path.join(REF, "*", "01_Si_band", "result", "a.log")))]
    bz = [b for b in bz if "mmm" in b and b.get("kpoints")]
    o2 = [parse_o2(p) for p in sorted(glob.glob(os.path.join(REF, "*", "02_O2-molecule_optimize", "*", "result", "a.log")))]
    o2 = [d for d in o2 if d.get("psv") and d.get("esp_scf1") and d.get("initrho")]
    o2_scf = [parse_o2_scf(p) for p in sorted(glob.glob(os.path.join(REF, "*", "02_O2-molecule_optimize", "*", "result", "a.log")))]
    o2_scf = [d for d in o2_scf if d.get("esp") and d["energies"].get("total") is not None]
    si = [parse_si(p) for p in sorted(glob.glob(os.path.join(REF, "*", "01_Si_band", "result", "a.log")))]
    si = [d for d in si if d.get("esp_scf1") and d["energies"].get("total") is not None]
    si_band = [parse_band_eigv(p) for p in sorted(glob.glob(os.path.join(REF, "*", "01_Si_band", "result", "band_eigv")))]
    si_band = [d for d in si_band if d["esp"]]
    json.dump({"kinetic": data, "bz": bz, "o2": o2, "o2_scf": o2_scf, "si": si, "si_band": si_band},
              open(os.path.join(HERE, "reference_logs.json"), "w"), indent=1)
    print(f"{len(data)} kinetic tables, {len(bz)} k-point lists, {len(o2)} O2 set-up/eigenvalue records, "
          f"{len(o2_scf)} converged O2 SCF records, {len(si)} Si records, {len(si_band)} Si band tables "
          f"-> reference_logs.json")


if __name__ == "__main__":
    main()
