/* Output-only stand-in for libcgns, used solely to compile the reference
 * solver as a test oracle. libcgns is not vendored with the reference and is
 * not installed here. Every call succeeds and writes nothing, so the solver's
 * arithmetic is untouched; only its CGNS output is dropped.
 * Covers the symbols used at zone_FD/src/src/block.cpp:11-56 and
 * zone_FD/src/src/cgnsio.cpp:3-101. */
#pragma once
typedef long cgsize_t;
enum { CG_MODE_READ = 0, CG_MODE_WRITE = 1, CG_MODE_MODIFY = 2 };
enum { CG_Structured = 2, CG_RealDouble = 4, CG_CellCenter = 3 };
#define CGNS_ENUMV(e) CG_##e
static inline int cg_open(const char *, int, int *fn) { *fn = 1; return 0; }
static inline void cg_error_exit(void) {}
static inline int cg_base_write(int, const char *, int, int, int *b) { *b = 1; return 0; }
static inline int cg_zone_write(int, int, const char *, const cgsize_t *, int, int *z) { *z = 1; return 0; }
static inline int cg_coord_write(int, int, int, int, const char *, const void *, int *c) { *c = 1; return 0; }
static inline int cg_sol_write(int, int, int, const char *, int, int *s) { *s = 1; return 0; }
static inline int cg_field_write(int, int, int, int, int, const char *, const void *, int *f) { *f = 1; return 0; }
static inline int cg_close(int) { return 0; }
