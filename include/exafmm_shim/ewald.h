/* Stands in for the reference's 3dp/ewald.h: the Ewald parts (wavePart, realPart,
 * selfTerm) and their globals, declared in exafmm_b200.hpp. */
#include "../exafmm_b200.hpp"
