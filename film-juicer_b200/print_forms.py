"""Runs the print exposure's spectral integral (fjb_print_raw) in one print form on the
capture density of the 3840x2160 synthetic frame, `--calls` times: the launch that an
ncu capture of one print-contraction kernel selects (profiles/print_forms_4k.md).

    python film-juicer_b200/print_forms.py --form tensor --calls 3
"""
from __future__ import annotations

import argparse
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--form", choices=["fp32", "tensor", "tensor_split"], default="tensor")
    ap.add_argument("--calls", type=int, default=3)
    ap.add_argument("--width", type=int, default=3840)
    ap.add_argument("--height", type=int, default=2160)
    args = ap.parse_args()
    import __graft_entry__

    __graft_entry__.package()
    import numpy as np
    import torch

    from film_juicer_b200 import abi, prepare, runtime

    code = {"fp32": abi.FJB_PRINT_FP32, "tensor": abi.FJB_PRINT_TENSOR,
            "tensor_split": abi.FJB_PRINT_TENSOR_SPLIT}[args.form]
    w, h = args.width, args.height
    recipe = prepare.PreparedRecipe.load(os.path.join(os.path.dirname(HERE), "tests", "golden", "recipe_print.npz"))
    dr = runtime.DeviceRecipe(prepare.HostRecord(recipe))
    src = torch.from_numpy(np.ascontiguousarray(prepare.synthetic_frame(w, h, seed=20261205))).cuda()
    dens = [torch.empty((h, w), device="cuda") for _ in range(3)]
    dr.capture_density(src, dens)
    raw = [torch.empty((h, w), device="cuda") for _ in range(3)]
    dr.set_print_form(code)
    for _ in range(args.calls):
        dr.print_raw(dens, raw)
    torch.cuda.synchronize()
    print(f"{args.form}: {args.calls} spectral integrals of {w}x{h}, mean raw M {float(raw[1].mean()):.6g}")
    dr.close()


if __name__ == "__main__":
    main()
