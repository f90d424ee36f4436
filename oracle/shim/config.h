/* Minimal config.h for compiling GSvit's CPU solver sources as the oracle.
 * Test infrastructure only.  UCUDA stays undefined: the reference GPU path is
 * not part of this build. */
#ifndef SHIM_CONFIG_H
#define SHIM_CONFIG_H
#define PACKAGE "gsvit"
#define VERSION "1.9.4"
#endif
