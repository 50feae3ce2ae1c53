/* declaration stub of <StgDomain/StgDomain.h>: see ../gale_stub.h */
#include "../gale_stub.h"
