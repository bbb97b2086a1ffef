"""Generates the golden fixtures under tests/golden/ from a copy of the reference tree.

Run once where the reference is available, naming its root (no default):
    python tests/golden/make_golden.py <reference_root>
    LEEDS_REFERENCE_ROOT=<reference_root> python tests/golden/make_golden.py
Outputs (committed):
  state_case1.cdf.gz  the reference's own tests/state.cdf.in (the Christensen case 1 state,
                      L=64, M=16, Mp=4, N=64, old-style dims uTH/uPH/BTH/BPH), byte for
                      byte, gzip-compressed with a fixed header (mtime 0) so that the
                      fixture is reproducible; tests read it through state.load_state;
  golden_case1.json   the first two rows (t = 0 and t = 4.59265755232e-6) of the reference's
                      time series for that state:
                      Benchmark_files/Boussinesq/Christensen_case1_benchmark/
                      vel_energy.dat and mag_energy.dat (columns as written there);
  planet_model_anelastic_benchmark.txt  the reference state of the anelastic benchmark
                      (Benchmark_files/Anelastic/Anelastic_benchmark/planet_model.txt.in,
                      128 shells, written by Scripts/anelastic_benchmark.m), copied verbatim.
"""
import gzip
import json
import os
import sys


def main(ref):
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(ref, "tests", "state.cdf.in"), "rb") as fh:
        raw = fh.read()
    with open(os.path.join(here, "state_case1.cdf.gz"), "wb") as out:
        with gzip.GzipFile(filename="state.cdf.in", mode="wb", compresslevel=9, fileobj=out, mtime=0) as gz:
            gz.write(raw)

    bdir = os.path.join(ref, "Benchmark_files", "Boussinesq", "Christensen_case1_benchmark")

    def rows(name, n):
        out = []
        with open(os.path.join(bdir, name)) as fh:
            for line in fh:
                if line.strip() and not line.lstrip().startswith("#"):
                    out.append([float(x) for x in line.split()])
                    if len(out) == n:
                        break
        return out

    vcols = ("time", "KE", "thermal", "topflx", "botflx", "KE_ax", "Edis")
    mcols = ("time", "ME", "dipole", "quadrupole", "ME_ax", "Mdis")
    vel, mag = rows("vel_energy.dat", 2), rows("mag_energy.dat", 2)
    golden = {
        "source": "Benchmark_files/Boussinesq/Christensen_case1_benchmark/{vel,mag}_energy.dat, rows 1-2",
        "vel_energy": [dict(zip(vcols, r)) for r in vel],
        "mag_energy": [dict(zip(mcols, r)) for r in mag],
    }
    with open(os.path.join(here, "golden_case1.json"), "w") as fh:
        json.dump(golden, fh, indent=1)
    src = os.path.join(ref, "Benchmark_files", "Anelastic", "Anelastic_benchmark", "planet_model.txt.in")
    with open(src) as fh, open(os.path.join(here, "planet_model_anelastic_benchmark.txt"), "w") as out:
        out.write(fh.read())
    print("wrote", sorted(os.listdir(here)))


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("LEEDS_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: make_golden.py <reference_root>  (or set LEEDS_REFERENCE_ROOT)")
    main(root)
