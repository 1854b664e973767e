"""Autotuner for the batched kernels' launch shapes.

Each k bin of the library has several compiled variants (threads per set,
i.e. warps per subset; sets per CTA; rows per thread; register cap; cluster
size for the large-k bins), listed by ``pl_tune_describe``.  ``tune()`` times
every variant of every bin on seeded synthetic sets at the bin's largest k and
writes the fastest per bin to a JSON file keyed by the GPU name;
``apply()`` selects those variants in the library (``pl_tune_set``).  The
library loads ``tuning.json`` next to this file automatically (or the file
named by ``PL_TUNING``) when it matches the current GPU.

    python -m paralanczos_b200.autotune [--out FILE] [--bins 0,1,...] [--seconds 0.05]
"""
from __future__ import annotations

import argparse
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_PATH = os.path.join(HERE, "tuning.json")


def _device_name() -> str:
    import torch
    return torch.cuda.get_device_name(torch.cuda.current_device())


def tune(bins=None, n: int = 4096, m: int = 2048, target_s: float = 0.05, reps: int = 2,
         out_path: str | None = DEFAULT_PATH, seed: int = 0, log=print) -> dict:
    """Time all variants of the given bins; returns (and writes) the choices."""
    import torch

    from . import api
    dev = torch.device("cuda", torch.cuda.current_device())
    g = torch.Generator(device=dev).manual_seed(seed)
    Phi = torch.randn(m, n, generator=g, device=dev, dtype=torch.float64) / m ** 0.5
    A = (Phi.T @ Phi).to(torch.float32).contiguous()
    del Phi
    nb = api.num_bins()
    bins = list(range(nb)) if bins is None else list(bins)
    result = {"device": _device_name(), "n": n, "m": m, "bins": {}}
    for b in bins:
        k = api.bin_kmax(b)
        nvar, _ = api.tune_describe(b, 0)
        # size the probe from a quick estimate with the current default
        api.tune_set(b, -1)
        probe = 256 if k > 128 else 4096
        idx = api.gen_sets(seed + 1, 0, probe, n, k)
        out = api.solve(A, idx, k=k)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        api.solve(A, idx, k=k, out=out)
        e1.record()
        torch.cuda.synchronize()
        rate = probe / max(e0.elapsed_time(e1) * 1e-3, 1e-6)
        nsets = int(min(max(rate * target_s, 512), 4_000_000))
        idx = api.gen_sets(seed + 1, 0, nsets, n, k)
        best = None
        times = []
        for v in range(nvar):
            api.tune_set(b, v)
            out = api.solve(A, idx, k=k)      # warm-up (loads the kernel, sizes scratch)
            torch.cuda.synchronize()
            e0.record()
            for _ in range(reps):
                api.solve(A, idx, k=k, out=out)
            e1.record()
            torch.cuda.synchronize()
            sps = nsets * reps / (e0.elapsed_time(e1) * 1e-3)
            desc = api.tune_describe(b, v)[1]
            times.append({"variant": v, "desc": desc, "sets_per_s": sps})
            if log:
                log(f"bin {b} (k<={k}) variant {v} [{desc}]: {sps:.3e} sets/s")
            if best is None or sps > best[1]:
                best = (v, sps, desc)
        api.tune_set(b, -1)
        result["bins"][str(b)] = {"kmax": k, "variant": best[0], "desc": best[2],
                                  "sets_per_s": best[1], "all": times}
    if out_path:
        with open(out_path, "w") as f:
            json.dump(result, f, indent=1)
    return result


def apply(path: str | None = None, lib=None) -> bool:
    """Select the tuned variants when the file matches the current GPU."""
    path = path or os.environ.get("PL_TUNING") or DEFAULT_PATH
    if not os.path.exists(path):
        return False
    try:
        with open(path) as f:
            data = json.load(f)
        import torch
        if not torch.cuda.is_available() or data.get("device") != _device_name():
            return False
    except Exception:
        return False
    import ctypes

    from . import _lib
    L = lib or _lib.lib()
    # entries are matched by the bin's k range and the variant's description,
    # so a file written by a build with other bins or variants still applies
    # to what it names (the rest keep their built-in defaults)
    bin_of = {L.pl_bin_kmax(b): b for b in range(L.pl_num_bins())}
    buf = ctypes.create_string_buffer(256)
    for ent in data.get("bins", {}).values():
        b = bin_of.get(int(ent.get("kmax", -1)))
        if b is None:
            continue
        nvar = L.pl_tune_describe(b, 0, buf, 256)
        for v in range(nvar):
            L.pl_tune_describe(b, v, buf, 256)
            if buf.value.decode() == ent.get("desc"):
                if L.pl_tune_set(b, v) != 0:
                    return False
                break
    return True


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_PATH)
    ap.add_argument("--bins", default="")
    ap.add_argument("--seconds", type=float, default=0.05)
    a = ap.parse_args()
    bins = [int(x) for x in a.bins.split(",") if x] or None
    tune(bins=bins, target_s=a.seconds, out_path=a.out)
    print("wrote", a.out)
    return 0


if __name__ == "__main__":
    sys.exit(main())
