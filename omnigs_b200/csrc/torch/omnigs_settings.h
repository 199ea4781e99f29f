// Settings of this package's LibTorch layer that the reference's interface has no place for
// (kept out of rasterize_points.h, which declares exactly the reference's functions).
#pragma once

// Transmittance checkpointing for the following RasterizeGaussiansCUDA calls of this process:
// the forward stores no per-pixel state (its imageBuffer holds only the tile ranges) and
// RasterizeGaussiansBackwardCUDA recomputes it (OMNIGS_FLAG_RECOMPUTE_T).  Off by default, which
// keeps the reference's stored final transmittance and last contributors.  The backward follows
// the mode of the forward that made its imageBuffer, whatever the setting is by then.
void omnigs_torch_set_recompute_transmittance(bool on);
bool omnigs_torch_recompute_transmittance();
