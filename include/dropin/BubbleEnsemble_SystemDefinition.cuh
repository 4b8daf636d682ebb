/* Drop-in stand-in for a driver's system-definition include: with libbes.so
 * the device callbacks are compiled into the library (BES_SYSTEM_DEFINITION
 * at build time; the Keller-Miksis collapse model by default), so the driver
 * side needs nothing here. */
#ifndef BES_DROPIN_SYSTEM_DEFINITION_CUH
#define BES_DROPIN_SYSTEM_DEFINITION_CUH
#endif
