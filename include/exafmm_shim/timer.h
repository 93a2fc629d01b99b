/* Stands in for the reference's 3d/timer.h: the driver API of minimal ExaFMM on the
 * GPU, declared in exafmm_b200.hpp (this directory goes on the include path
 * before the reference's own headers). */
#include "../exafmm_b200.hpp"
