/* Minimal configure.h for compiling the reference's standalone *_impl.h
 * kernels on the host (oracle/_ref build only): legacy Athena++ indexing
 * off, host-only dispatch. */
#pragma once
#define NMASS 0
#define DISPATCH_MACRO
