"""Tuner of the patch solvers' launch parameters for the current GPU model.

Times whole transfers (CUDA events, median after warm-up, inputs resident on
the device) over these parameters, by coordinate descent from the built-in
defaults:

* ``PACMAN_B200_INT8_FROM``: the first tile column whose update runs on the
  int8 tensor cores (the columns before it use the FP64 tensor cores);
* ``PACMAN_B200_GROUPS``: slot groups of the tiled engine, each stepping on
  its own stream;
* ``PACMAN_B200_BIG_N``: patches above this size use the tiled Cholesky
  instead of the register kernels (at most 64);
* ``PACMAN_B200_BACK_STAGES``: ring depth (3 or 6) of the one-field
  backward sweep.

The library reads each parameter per call from the environment, so the
tuner sets them there.  With ``--write`` the best choice goes to
``tuning/<GPU name>.conf`` beside ``libpacman_b200.so``, which the library
reads once per device; an environment variable still overrides it.

    python -m pacman_b200.tune --workload grid_blobs_1m --write
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import sys

SPACE = {
    "PACMAN_B200_INT8_FROM": ["0", "1", "2", "3", "4", "5", "6"],
    "PACMAN_B200_GROUPS": ["1", "2", "3", "4", "6", "8"],
    "PACMAN_B200_BIG_N": ["32", "48", "64"],
    "PACMAN_B200_BACK_STAGES": ["3", "6"],
}
DEFAULTS = {"PACMAN_B200_INT8_FROM": "4", "PACMAN_B200_GROUPS": "4",
            "PACMAN_B200_BIG_N": "64", "PACMAN_B200_BACK_STAGES": "3"}


def conf_path(device_name: str) -> str:
    here = os.path.dirname(os.path.abspath(__file__))
    stem = re.sub(r"[^A-Za-z0-9.\-]", "_", device_name)
    return os.path.join(here, "tuning", stem + ".conf")


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--workload", default="grid_blobs_1m")
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--passes", type=int, default=2)
    ap.add_argument("--write", action="store_true")
    args = ap.parse_args(argv)

    import torch

    import pacman_b200 as pacman
    from pacman_b200 import workloads as W

    dev = torch.device("cuda", 0)
    w = W.make(args.workload, args.scale)
    S = torch.tensor(w["src"], device=dev)
    T = torch.tensor(w["tgt"], device=dev)
    V = torch.tensor(w["values"][:, 0] if w["values"].shape[1] == 1 else w["values"], device=dev)

    def run(cfg):
        for k, v in cfg.items():
            os.environ[k] = v
        times, st = [], {}
        for i in range(args.reps + 2):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            pacman.rbf.interpolate(3, pacman.execspaces.CUDA, w["basis"], S, V, T,
                                   nodes_per_cluster=w["nodes_per_cluster"], precision="mixed",
                                   stats=st)
            e1.record()
            e1.synchronize()
            if i >= 2:
                times.append(e0.elapsed_time(e1))
        return statistics.median(times), st

    log = []
    best = dict(DEFAULTS)
    best_ms, best_st = run(best)
    log.append({"config": dict(best), "ms": best_ms})
    for _ in range(args.passes):
        improved = False
        for key, values in SPACE.items():
            for v in values:
                if v == best[key]:
                    continue
                cfg = dict(best, **{key: v})
                ms, st = run(cfg)
                log.append({"config": cfg, "ms": ms})
                if ms < best_ms * 0.99:
                    best, best_ms, best_st, improved = cfg, ms, st, True
        if not improved:
            break
    for k in SPACE:
        os.environ.pop(k, None)
    name = torch.cuda.get_device_name(dev)
    result = {"device": name, "workload": args.workload, "scale": args.scale, "best": best,
              "best_ms": best_ms, "default_ms": log[0]["ms"],
              "kernel_launches": best_st.get("kernel_launches"),
              "host_syncs": best_st.get("host_syncs"), "tried": log}
    print(json.dumps(result))
    if args.write:
        path = conf_path(name)
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path, "w") as f:
            f.write(f"# Launch parameters for {name}, chosen by python -m pacman_b200.tune\n")
            f.write(f"# on {args.workload} (scale {args.scale}): {best_ms:.2f} ms per transfer "
                    f"(built-in defaults: {log[0]['ms']:.2f} ms), median of {args.reps}.\n")
            for k, v in best.items():
                f.write(f"{k} = {v}\n")
        print(path, file=sys.stderr)
    return 0


if __name__ == "__main__":
    sys.exit(main())
