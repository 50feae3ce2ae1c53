/* declaration stub of <StGermain/StGermain.h>: see ../gale_stub.h */
#include "../gale_stub.h"
