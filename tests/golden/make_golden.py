"""Extract the reference's own known-answer files for the NEGF recursion.

The reference ships three standalone RGF programs whose outputs are committed
in its tree.  This script copies the numeric tables (data only, no source)
into ``tests/golden/`` so that the tests can run where the reference tree is
absent.  It reads the reference checkout given by ``--ref`` or, failing that,
by the ELEQTRONEX_REFERENCE environment variable; there is no default path.

    python tests/golden/make_golden.py --ref <path of the reference checkout>

  decimation_technique/Exec/output/{Sigma,DOS,Transmission}
      N=4, 10 energies on [-6, 0] + 1e-8 i, beta = 2*2.5*cos(6 pi/17),
      surface GF root (F - S)/D  (scripts/negf_cpp/decimation_technique/Source/main.cpp)
  negf_python/PointContact/cpp_results/1gpu/{Sigma,DOS,Transmission}
      N=4, 1000 energies on [-1, 1] + 1e-8 i, root (F + S)/D
      (scripts/negf_cpp/spectral_function_1D_pll/Source/main.cpp)
  negf_python/DOS_Compare/cpp_results/gpu/{LDOS,Transmission}.dat
      output of the engine's own Compute_DensityOfStates for a (17,0) CNT of
      one unit cell (N=4), 2 modes, analytic leads, 200 uniform energies on
      [-1, 1] + 1e-8 i: DOS per unit cell and transmission per energy
"""
import argparse
import os
import shutil

SETS = {
    "decimation": "scripts/negf_cpp/decimation_technique/Exec/output",
    "pointcontact_1gpu": "scripts/negf_python/PointContact/cpp_results/1gpu",
}
FILES = ["Sigma", "DOS", "Transmission"]
DOS_COMPARE = ("scripts/negf_python/DOS_Compare/cpp_results/gpu", ["LDOS.dat", "Transmission.dat"])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("ELEQTRONEX_REFERENCE"),
                    help="reference checkout (default: $ELEQTRONEX_REFERENCE)")
    args = ap.parse_args()
    if not args.ref:
        ap.error("give the reference checkout with --ref or ELEQTRONEX_REFERENCE")
    here = os.path.dirname(os.path.abspath(__file__))
    for tag, rel in SETS.items():
        for f in FILES:
            src = os.path.join(args.ref, rel, f)
            dst = os.path.join(here, f"{tag}_{f}.txt")
            shutil.copyfile(src, dst)
            print(f"{src} -> {dst}")
    rel, files = DOS_COMPARE
    for f in files:
        src = os.path.join(args.ref, rel, f)
        dst = os.path.join(here, "dos_compare_gpu_" + f.replace(".dat", ".txt"))
        shutil.copyfile(src, dst)
        print(f"{src} -> {dst}")


if __name__ == "__main__":
    main()
