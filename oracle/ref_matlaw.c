/* ref_matlaw.c -- test infrastructure for oracle/_ref (never shipped).
 *
 * The reference's membmodel.c reads the Fortran COMMON block /MATLAW/
 * (membmodel.c:14-18, common.f90:4) as `extern struct {double hf_gscell;}`.
 * Compiled with -DUNDERSCORE the symbol is `matlaw_`.  This file provides that
 * block and a setter so the unmodified membmodel.c can be called from ctypes
 * to pin the oracle's restated Skalak law. */
struct { double hf_gscell; } matlaw_;

void ref_set_hf_gscell(double v) { matlaw_.hf_gscell = v; }
