"""Prints the FP32-vs-FP64 error table of one solver (both precision modes)
as markdown; test infrastructure (it drives the FP64 oracle).

    python tests/precision_report.py --n-side 1024 --steps 1000 --at 1,10,1000
    python tests/precision_report.py --method iisph --n-side 256 --steps 100 --at 1,10,100
"""
import argparse
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n-side", type=int, default=1024)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--at", default="1,10,1000")
    ap.add_argument("--method", default="dfsph_p",
                    choices=("dfsph_p", "iisph", "iisph_ap", "iisph_pseudo_ap", "pcisph"))
    args = ap.parse_args()
    import emerald_b200 as E
    from precision import compare
    at = {int(s) for s in args.at.split(",")}
    print("%s dam break %dx%d (%d particles), dx = 1/%d, support = dx; FP32 run vs the FP64 "
          "GPU oracle with the same sub-steps and iteration counts\n" % (
              args.method.upper(), args.n_side, args.n_side, args.n_side ** 2, 2 * args.n_side))
    print("| mode | sub-step | density err L_inf | density err RMS | position err max (dx) | "
          "position err RMS (dx) | position err p99 (dx) | kinetic energy rel. diff | "
          "energy drift FP32 | energy drift FP64 | particles > 50 m/s FP32 / FP64 | "
          "iterations |")
    print("|---|---:|---:|---:|---:|---:|---:|---:|---:|---:|---:|---:|")
    for name, mode in (("reference FP32", E.PRECISION_REFERENCE),
                       ("compensated", E.PRECISION_COMPENSATED)):
        t0 = time.time()
        rows = compare(E, args.n_side, args.steps, at, mode, method=args.method)
        for r in rows:
            print("| %s | %d | %.3e | %.3e | %.3e | %.3e | %.3e | %.3e | %.3e | %.3e | %d / %d | "
                  "%d |" % (
                      name, r["step"], r["density_linf"], r["density_rms"], r["position_max_dx"],
                      r["position_rms_dx"], r["position_p99_dx"], r["energy_rel_diff"],
                      r["energy_drift"], r["energy_drift_fp64"], r["fast_fp32"], r["fast_fp64"],
                      r["iterations"]), flush=True)
        print("<!-- %s: %.1f s -->" % (name, time.time() - t0), flush=True)


if __name__ == "__main__":
    main()
