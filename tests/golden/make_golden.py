"""Extract golden values for the PM7 SCF path from the reference's own tests.

Usage: python tests/golden/make_golden.py <reference checkout>

It writes tests/golden/reference_values.json.  Sources (paths inside the
reference checkout):
  tests/keywords/1SCF.mop / 1SCF.out   CO2 PM7 1SCF: heat (:70), eigenvalues
                                       (:118-120), net charges (:125-127)
  tests/keywords/VECTORS.mop / .out    propane PM7 (first job): heat (:91),
                                       eigenvalues (:156-159), charges (:164-174)
  tests/mopac_api_test.F90:61-104      H2O PM7 SCF: heat, charges
  tests/mopac_api_test.F90:379-454     the same H2O through MOZYME: heat, charges
"""
import json
import os
import re
import sys

if len(sys.argv) != 2:
    sys.exit("usage: python tests/golden/make_golden.py <reference checkout>")
REF = sys.argv[1]
SYM = {"H": 1, "C": 6, "O": 8}


def parse_out(path):
    lines = open(path).read().splitlines()
    out = {}
    for i, l in enumerate(lines):
        if "FINAL HEAT OF FORMATION" in l and "heat" not in out:
            out["heat"] = float(l.split("=")[1].split()[0])
        if l.strip() == "EIGENVALUES" and "eigs" not in out:
            vals = []
            j = i + 1
            while lines[j].strip():
                vals += [float(x) for x in lines[j].split()]
                j += 1
            out["eigs"] = vals
        if "NET ATOMIC CHARGES AND DIPOLE" in l and "charges" not in out:
            q = []
            j = i + 3
            while lines[j].strip() and not lines[j].startswith(" DIPOLE"):
                q.append(float(lines[j].split()[2]))
                j += 1
            out["charges"] = q
    return out


def parse_mop_first(path):
    lines = open(path).read().splitlines()
    nat, xyz = [], []
    for l in lines[3:]:
        a = l.split()
        if not a:
            break
        nat.append(SYM[a[0]])
        xyz.append([float(a[1]), float(a[2]), float(a[3])])
    return nat, xyz


g = {}
nat, xyz = parse_mop_first(os.path.join(REF, "tests/keywords/1SCF.mop"))
g["co2_1scf"] = dict(nat=nat, xyz=xyz, **parse_out(os.path.join(REF, "tests/keywords/1SCF.out")),
                     source="tests/keywords/1SCF.out")
nat, xyz = parse_mop_first(os.path.join(REF, "tests/keywords/VECTORS.mop"))
g["propane"] = dict(nat=nat, xyz=xyz, **parse_out(os.path.join(REF, "tests/keywords/VECTORS.out")),
                    source="tests/keywords/VECTORS.out")
src = open(os.path.join(REF, "tests/mopac_api_test.F90")).read()
blk = src[src.index("subroutine test_mopac_scf1"):src.index("end subroutine test_mopac_scf1")]
coord = [float(m) for m in re.findall(r"test_in%coord\(\d\) = (-?[\d.]+)d0", blk)]
heat = float(re.search(r"test_target%heat = (-?[\d.]+)d0", blk).group(1))
charge = [float(m) for m in re.findall(r"test_target%charge\(\d\) = (-?[\d.]+)d0", blk)]
g["h2o_api"] = dict(nat=[1, 1, 8], xyz=[coord[0:3], coord[3:6], coord[6:9]], heat=heat, charges=charge,
                    source="tests/mopac_api_test.F90:61-104")
blk = src[src.index("subroutine test_mozyme_scf1"):src.index("end subroutine test_mozyme_scf1")]
coord = [float(m) for m in re.findall(r"test_in%coord\(\d\) = (-?[\d.]+)d0", blk)]
heat = float(re.search(r"test_target%heat = (-?[\d.]+)d0", blk).group(1))
charge = [float(m) for m in re.findall(r"test_target%charge\(\d\) = (-?[\d.]+)d0", blk)]
g["h2o_mozyme"] = dict(nat=[1, 1, 8], xyz=[coord[0:3], coord[3:6], coord[6:9]], heat=heat, charges=charge,
                       source="tests/mopac_api_test.F90:379-454")
json.dump(g, open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_values.json"), "w"),
          indent=1)
print({k: len(v.get("eigs", [])) for k, v in g.items()})
