/* declaration stub of <StgFEM/StgFEM.h>: see ../gale_stub.h */
#include "../gale_stub.h"
