/*
 * posix_shim.h - Forced include (g++ -include) that lets the reference's CPU sources build on Linux.
 *
 * Test infrastructure only: it is used by oracle/Makefile when it compiles the reference's own
 * CPU variant (src/common, src/cpu, src/cli of acesds/sadcs) into oracle/_ref/. The reference
 * targets Windows and calls three MSVC CRT names; each maps onto its POSIX equivalent here.
 * The reference sources themselves are compiled unchanged, where they lie.
 */
#pragma once

#include <stdio.h>
#include <stdlib.h>
#include <sys/types.h>

#define _fseeki64 fseeko
#define _ftelli64 ftello
#define _putenv_s(name, value) setenv((name), (value), 1)
