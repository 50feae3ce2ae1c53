/* declaration stub of <PICellerator/PICellerator.h>: see ../gale_stub.h */
#include "../gale_stub.h"
