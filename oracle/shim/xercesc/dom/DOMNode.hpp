// Xerces-C header name mapped onto the oracle DOM shim (test infrastructure).
#include "../grains_dom_shim.hpp"
