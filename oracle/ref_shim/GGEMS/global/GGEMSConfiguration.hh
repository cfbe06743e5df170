// Test infrastructure only: stand-in for the header CMake generates from the
// reference's cmake-config/GGEMSConfiguration.hh.in (CMakeLists.txt:128-132),
// with the reference's default MAXIMUM_PARTICLES.  Used solely to compile the
// reference's device kernels through oracle/ref_shim/ocl_shim.hh.
#ifndef GUARD_GGEMS_GLOBAL_GGEMSCONFIGURATION_HH
#define GUARD_GGEMS_GLOBAL_GGEMSCONFIGURATION_HH
#define MAXIMUM_PARTICLES 1048576
#endif
