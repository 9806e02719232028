// Compiles the reference's own obstacles/Obstacle.cpp, unmodified, against the
// stand-ins of oracle/ref_shim (test infrastructure of the oracle only).
#define CUP_NO_MACROS_HEADER
#include "obstacles/Obstacle.cpp"
