/* TEST INFRASTRUCTURE ONLY -- CPU oracle for the primary-Compton scatter sysmat (filled in below). */
#include "oracle_common.h"
