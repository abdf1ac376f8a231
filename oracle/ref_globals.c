/* TEST ORACLE ONLY: instantiates the reference's global variables by
 * including its globvar.h (compiled in place from the reference tree). */
#include "fd.h"
#include "globvar.h"
