/*
 * start.h -- initialisation and geometry helpers (plqcd-b200).
 *
 * Same entry points as the reference's include/start.h:30-87
 * (implementations lib/start.c:19-247, 255-526, 1169-1428). Error
 * behaviour differs on purpose: where the reference prints and calls
 * exit(1), these functions return an error code (or -1) and record the
 * message for plqcd_last_error() (include/plqcd_b200.h). They never
 * terminate the caller.
 */
#ifndef _START_H
#define _START_H

#include "plqcd_global_params.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Read the key-value input file argv[1] (keys L0..L3, NPROC0..3, NTHREAD,
 * ALIGN; lib/start.c:84-107), validate it (extents even and >= 4, one
 * process in every direction), build the geometry tables and bind the CUDA
 * device (PLQCD_DEVICE, default 0; without a device the host-side API
 * still works). Returns 0 on success, 0 again if already initialised,
 * non-zero on failure. */
int init_plqcd(int argc, char *argv[]);

/* Release the tables and every device resource of the drop-in path. */
void finalize_plqcd(void);

/* Process index of grid coordinates n[] (lib/start.c:1169-1183); -1 when
 * out of range. */
int ipr(int n[]);

/* Grid coordinates of process ip (lib/start.c:1190-1212). */
void comp_cpr(int ip, int n[]);

/* Neighbour process ids into plqcd_g.npr (lib/start.c:1227-1248). */
void set_npr(void);

/* Local coordinates of lexicographic index ix (lib/start.c:1256-1270);
 * x fastest. Leaves xcor untouched when ix is out of range. */
void lex2cart(int ix, int xcor[]);

/* Lexicographic index of local coordinates (lib/start.c:1278-1298); -1 when
 * a coordinate is out of range. */
int cart2lex(int xcor[]);

/* Build ipt_eo, ipt_lex, iup, idn, face and the yzt block tables from
 * plqcd_g.latdims (lib/start.c:255-560). */
void set_geometry(void);

/* Process id and even/odd index of global coordinates xg[]
 * (lib/start.c:1308-1343); *pid = -1 when out of range. */
void find_site(int xg[], int *pid, int *xeo);

/* Print the contents of plqcd_g (lib/start.c:1351-1428, same format). */
void print_params(FILE *fp);

#ifdef __cplusplus
}
#endif
#endif
