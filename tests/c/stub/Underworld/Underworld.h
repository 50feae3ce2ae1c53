/* declaration stub of <Underworld/Underworld.h>: see ../gale_stub.h */
#include "../gale_stub.h"
