// Stand-in for the reference's src/Textures.h (legacy texture references, which CUDA 12
// no longer compiles).  The headers the pin harness includes declare but never read those
// textures, so nothing is needed here.  Test infrastructure only.
#pragma once
