/* Drop-in replacement for the reference's include/Falcons/api/falcons.hpp: callers that include
 * "Falcons/api/falcons.hpp" with this directory ahead of the reference's include directory get the
 * same API with the B200 library underneath (see falcons_gpu.hpp). */
#ifndef Falcons_Falcons_HPP
#define Falcons_Falcons_HPP
#include "falcons_gpu.hpp"
#endif
