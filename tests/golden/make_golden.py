"""Generates the golden fixtures under tests/golden/ from the reference tree.

Run once in a container where the reference is mounted (default /root/reference):
    python tests/golden/make_golden.py [reference_root]
Outputs (committed):
  state_case1.npz   the coefficients of the reference's tests/state.cdf.in
                    (L=64, M=16, Mp=4, N=64; variables uT,uP,C,BT,BP as (2,544,64)
                    and the radial grid r, dt, t), copied verbatim;
  golden_t0.json    the t=0 rows of the reference's own time series for that state:
                    Benchmark_files/Boussinesq/Christensen_case1_benchmark/
                    vel_energy.dat and mag_energy.dat (columns as written there);
  planet_model_anelastic_benchmark.txt  the reference state of the anelastic benchmark
                    (Benchmark_files/Anelastic/Anelastic_benchmark/planet_model.txt.in,
                    128 shells, written by Scripts/anelastic_benchmark.m), copied verbatim.
"""
import json
import os
import sys

import numpy as np
from scipy.io import netcdf_file

ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
here = os.path.dirname(os.path.abspath(__file__))

f = netcdf_file(os.path.join(ref, "tests", "state.cdf.in"), "r", mmap=False)
arrs = {k: np.array(f.variables[k].data, dtype=np.float64) for k in ("uT", "uP", "C", "BT", "BP")}
attrs = {k: int(f.variables["uT"]._attributes[k]) for k in ("L", "M", "Mp")}
np.savez_compressed(os.path.join(here, "state_case1.npz"),
                    r=np.array(f.variables["r"].data, dtype=np.float64),
                    dt=float(f.variables["dt"].data), t=float(f._attributes["t"]),
                    L=attrs["L"], M=attrs["M"], Mp=attrs["Mp"],
                    E=float(f._attributes["E"]), Ra=float(f._attributes["Ra"]),
                    Pr=float(f._attributes["Pr"]), Pm=float(f._attributes["Pm"]),
                    riro=float(f._attributes["riro"]), **arrs)
f.close()

bdir = os.path.join(ref, "Benchmark_files", "Boussinesq", "Christensen_case1_benchmark")
def first_row(name):
    with open(os.path.join(bdir, name)) as fh:
        for line in fh:
            if line.strip() and not line.lstrip().startswith("#"):
                return [float(x) for x in line.split()]
vel = first_row("vel_energy.dat")
mag = first_row("mag_energy.dat")
golden = {
    "source": "Benchmark_files/Boussinesq/Christensen_case1_benchmark/{vel,mag}_energy.dat, t=0 row",
    "vel_energy_t0": {"time": vel[0], "KE": vel[1], "thermal": vel[2], "topflx": vel[3],
                      "botflx": vel[4], "KE_ax": vel[5], "Edis": vel[6]},
    "mag_energy_t0": {"time": mag[0], "ME": mag[1], "dipole": mag[2], "quadrupole": mag[3],
                      "ME_ax": mag[4], "Mdis": mag[5]},
}
with open(os.path.join(here, "golden_t0.json"), "w") as fh:
    json.dump(golden, fh, indent=1)
src = os.path.join(ref, "Benchmark_files", "Anelastic", "Anelastic_benchmark", "planet_model.txt.in")
with open(src) as fh, open(os.path.join(here, "planet_model_anelastic_benchmark.txt"), "w") as out:
    out.write(fh.read())
print("wrote", os.listdir(here))
