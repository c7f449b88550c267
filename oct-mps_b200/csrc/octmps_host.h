// Internal declarations shared by the host-side sources of the library.
#ifndef OCTMPS_HOST_H
#define OCTMPS_HOST_H

#include "octmps_capi.h"

#endif
