// Empty stand-in: the reference's cpu_kernels.hpp includes a PD3_types.hpp
// that is not part of its source tree; nothing from it is used.
#pragma once
