/*
 * plqcd.h -- umbrella header (plqcd-b200), as the reference's
 * include/plqcd.h:17-18: initialisation, geometry and the hopping matrix,
 * plus the device-resident extensions of plqcd_b200.h.
 */
#ifndef _PLQCD_H
#define _PLQCD_H
#include "start.h"
#include "dirac.h"
#include "plqcd_b200.h"
#endif
