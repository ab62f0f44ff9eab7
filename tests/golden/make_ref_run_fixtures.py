"""Copy the reference's committed TreePM stepping runs at one rank into
tests/golden/ref_runs/: each run's TOML config and its per-step
diagnostics.jsonl (kinetic energy, momentum, angular momentum, centre of mass,
v_rms, delta_rms, a), written by gadget-ng's own `run` command.  They pin the
oracle's initial conditions, PM, short-range walk, KDK step and cosmology to
reference outputs.  Run once in a checkout that has the reference tree:
    python tests/golden/make_ref_run_fixtures.py <gadget-ng checkout root>
"""
import os
import shutil
import sys

RUNS = {
    # name: (config, results directory), both under experiments/nbody/
    "eds_N512": ("phase23_sr_sfc_domain/configs/eds_N512_sr_sfc_p1.toml",
                 "phase23_sr_sfc_domain/results/fase23_sr_sfc_p1"),
    "eds_N1000": ("phase25_mpi_validation/configs/eds_N1000_fase23.toml",
                  "phase25_mpi_validation/results/fase23_N1000_P1"),
    "lcdm_N2000": ("phase25_mpi_validation/configs/lcdm_N2000_fase23.toml",
                   "phase25_mpi_validation/results/fase23_N2000_P1"),
}
DST = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_runs")


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_ref_run_fixtures.py <gadget-ng checkout root>")
    root = os.path.join(sys.argv[1], "experiments", "nbody")
    os.makedirs(DST, exist_ok=True)
    for name, (cfg, res) in RUNS.items():
        shutil.copyfile(os.path.join(root, cfg), os.path.join(DST, name + ".toml"))
        shutil.copyfile(os.path.join(root, res, "diagnostics.jsonl"), os.path.join(DST, name + ".diagnostics.jsonl"))


if __name__ == "__main__":
    main()
