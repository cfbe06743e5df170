// Test infrastructure only: stand-in for the export header the reference's
// CMake build generates; the shim build exports nothing.
#ifndef GUARD_GGEMS_GLOBAL_GGEMSEXPORT_HH
#define GUARD_GGEMS_GLOBAL_GGEMSEXPORT_HH
#define GGEMS_EXPORT
#endif
