"""Regenerate dalton_energies.json from Dalton's stored test outputs.

Reads the golden numbers as text from a Dalton source tree (its path is the
one argument) and writes them, with their file:line provenance, into
tests/golden/dalton_energies.json.  The tests read only the JSON.

    python tests/golden/make_golden.py <path to a Dalton source tree>
"""
import json
import os
import re
import sys

SRC = sys.argv[1] if len(sys.argv) > 1 else None
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "dalton_energies.json")


def lines(rel):
    with open(os.path.join(SRC, rel), errors="replace") as f:
        return f.read().splitlines()


def grab_float(text):
    return float(re.findall(r"-?\d+\.\d+", text)[-1])


def main():
    ed = lines("DALTON/test/trueresult/energy_direct.ref")
    ac_rel = "DALTON/test/geoopt_preopt2/result/preopt_acrolein.out"
    ac = lines(ac_rel)
    adz = lines("DALTON/test/trueresult/benchmark_her_adz.ref")
    assert "Final HF energy" in ed[658] and "Nuclear repulsion energy" in ed[414]
    coords = []
    for ln in ac[334:342]:
        v = re.findall(r"-?\d+\.\d+", ln)
        coords.append([float(x) for x in v[:3]])
    grad = [[float(x) for x in re.findall(r"-?\d+\.\d+", ln)[:3]] for ln in ac[842:850]]
    assert "Final HF energy" in ac[636] and len(grad) == 8
    g = {
        "energy_direct": {"source": "DALTON/test/trueresult/energy_direct.ref:415,659 "
                                    "(input DALTON/test/energy_direct:30-43)",
                          "basis": "cc-pVDZ", "energy": grab_float(ed[658]), "nuclear_repulsion": grab_float(ed[414])},
        "preopt_acrolein": {"source": f"{ac_rel}:331-342,637,840-850 (input acrolein.mol); gradient rows 843-850", "basis": "STO-3G",
                            "energy": grab_float(ac[636]), "coords_bohr": coords, "gradient": grad},
        "benchmark_her_adz": {"source": "DALTON/test/trueresult/benchmark_her_adz.ref:853", "basis": "aug-cc-pVDZ",
                              "energy": grab_float(adz[852]),
                              "note": "Bz-H2 complex; geometry in DALTON/test/benchmark_her_adz:30-62 "
                                      "(not used by the tests yet)"},
    }
    with open(OUT, "w") as f:
        json.dump(g, f, indent=1)
    print("wrote", OUT)


if __name__ == "__main__":
    if SRC is None:
        sys.exit("usage: make_golden.py <path to a Dalton source tree>")
    main()
