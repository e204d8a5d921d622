// The wavefront RIS kernels with the closures' texture overrides
// (PreviewSurfaceMaterial::GetClosure, preview_surface.cpp:68-95), as
// hdr::textured::launch_*: the host launches these for scenes with textures.
#define HDR_WAVE_TEXTURED 1
#define HDR_TEXTURES 1
#include "wavefront.cu"
