// Empty stand-in for the CUDA header the reference kernel includes; the
// emulation shim provides everything the kernel uses.
#pragma once
