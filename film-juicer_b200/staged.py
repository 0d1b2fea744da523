"""A frame rendered one library call per stage, for precision reports and debugging:
the stages fj_cuda_render schedules for a frame with camera exposure, camera
diffusion, scatter/halation, spatial DIR, grain and the scan, in the reference's
staged order (src/Cuda/JuicerCudaExecutor.cpp:1874-2400; fjb_schedule.cpp), each fed
the previous stage's device planes, with every intermediate copied back to the host."""
from __future__ import annotations

from . import abi, runtime


def render_staged(record, src):
    """A frame's stages one library call at a time, each fed the previous
    stage's device planes (so errors accumulate as in the fused frame): the carrier after
    camera exposure, camera diffusion and scatter/halation (B, G, R), the spatial-DIR
    filtered corrections (Y, M, C), the capture density and the grained density (C, M, Y),
    and the encoded output. Returns host copies by stage name."""
    import torch

    h = record.host.h
    unsupported = (h.film_exposure.flags & abi.FJ_FILM_AUTO_EXPOSURE or
                   h.optics.flags & (abi.FJ_OPTICS_HIGHLIGHT_BOOST | abi.FJ_OPTICS_ENLARGER_DIFFUSION) or
                   h.effects.flags & (abi.FJ_EFFECTS_FILM | abi.FJ_EFFECTS_GATE_OUTPUT))
    if unsupported:
        raise RuntimeError("the staged precision chain covers exposure, diffusion, scatter/halation, "
                           "spatial DIR, grain and the scan")
    H, W = src.shape[0], src.shape[1]
    out = {}

    def keep(name, planes):
        torch.cuda.synchronize()
        out[name] = [t.cpu().numpy().copy() for t in planes]

    plane = lambda: torch.empty((H, W), device="cuda", dtype=torch.float32)
    dr = runtime.DeviceRecipe(record.host)
    try:
        carrier = [plane() for _ in range(3)]  # B, G, R
        dr.camera_exposure(src, carrier)
        keep("camera_exposure", carrier)
        if h.optics.flags & abi.FJ_OPTICS_CAMERA_DIFFUSION:
            d = h.optics.camera
            diffused = [plane() for _ in range(3)]
            runtime.diffusion(runtime.diffusion_components(d), d.radius_px, d.scatter_fraction,
                              [carrier[2], carrier[1], carrier[0]], [diffused[2], diffused[1], diffused[0]])
            carrier = diffused
            keep("camera_diffusion", carrier)
        if h.optics.flags & abi.FJ_OPTICS_SCATTER_HALATION:
            runtime.scatter_halation(h.optics.scatter_halation, [carrier[2], carrier[1], carrier[0]])
            keep("scatter_halation", carrier)
        density = [plane() for _ in range(3)]  # C, M, Y
        if h.spatial_dir.component_count > 0:
            filtered = [plane() for _ in range(3)]
            log_raw = [plane() for _ in range(3)]
            dr.spatial_dir_build(h.spatial_dir, filtered, log_raw, carrier=carrier)
            keep("spatial_dir_filtered", filtered)
            dr.set_spatial_dir_planes(filtered, log_raw)
        dr.capture_density(None, density, carrier=carrier)
        dr.set_spatial_dir_planes(None)
        keep("capture_density", density)
        if h.grain.flags & abi.FJ_GRAIN_ACTIVE:
            noise = runtime.DeviceNoise(record.noise.record) if record.noise is not None else None
            runtime.visual_grain(dr, h.grain, density, noise)
            keep("grain", density)
            if noise is not None:
                noise.close()
        dst = torch.empty_like(src)
        dr.render_from_density(density, src, dst)
        torch.cuda.synchronize()
        out["output"] = dst.cpu().numpy()
    finally:
        dr.close()
    return out
