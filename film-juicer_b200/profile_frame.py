"""Renders `--frames` full optical print frames (every spatial stage on, the bench's
recipe and synthetic scene) through fj_cuda_render, for ncu captures of single kernels
and launch lists of the frame (profiles/*.md give the exact commands).

    python film-juicer_b200/profile_frame.py --width 1920 --height 1080 --frames 2
"""
from __future__ import annotations

import argparse
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--frames", type=int, default=2)
    ap.add_argument("--print-form", choices=["fp32", "tensor", "tensor_split"], default="fp32")
    ap.add_argument("--next-rows", action="store_true",
                    help="add highlight reconstruction, scanner post effects and film / gate defects with weave "
                         "(the bench's --next-rows frame)")
    args = ap.parse_args()
    import __graft_entry__

    __graft_entry__.package()
    import numpy as np
    import torch

    from film_juicer_b200 import abi, frame_records, prepare, runtime

    w, h = args.width, args.height
    recipe = prepare.PreparedRecipe.load(os.path.join(os.path.dirname(HERE), "tests", "golden", "recipe_print.npz"))
    if args.next_rows:
        from film_juicer_b200 import descriptors

        record = frame_records.FrameRecord(
            recipe, w, h, highlight_boost=descriptors.highlight_boost_record(4.0, 3.0, 1.5),
            post=descriptors.scanner_post_record(glare_percent=0.3, glare_roughness=0.4, glare_blur_sigma_px=4.0,
                                                 lens_blur_sigma_px=0.8, unsharp_sigma_px=0.7, unsharp_amount=0.7),
            effects=descriptors.default_film_effects(w, h))
    else:
        record = frame_records.FrameRecord(recipe, w, h)
    src = torch.from_numpy(np.ascontiguousarray(prepare.synthetic_frame(w, h, seed=20261205))).cuda()
    dst = torch.empty_like(src)
    form = {"fp32": abi.FJB_PRINT_FP32, "tensor": abi.FJB_PRINT_TENSOR,
            "tensor_split": abi.FJB_PRINT_TENSOR_SPLIT}[args.print_form]
    with runtime.Owner() as owner:
        owner.set_print_form(form)
        for _ in range(args.frames):
            owner.render(record, src, dst)
        torch.cuda.synchronize()
    print(f"{args.frames} frames of {w}x{h}, output mean {float(dst.mean()):.6g}")


if __name__ == "__main__":
    main()
