/* Single-rank stand-in for the MPI API, used only to compile the reference's
 * CPU code (BetterTT06, FGRDiffusionOMP, singleCell, the object database)
 * into the oracle.  Every collective is the identity on one rank.  Test
 * infrastructure: nothing in the product links this. */
#ifndef ORACLE_REF_MPI_STUB_H
#define ORACLE_REF_MPI_STUB_H
#include <string.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef long MPI_Aint;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
#define MPI_COMM_WORLD 0
#define MPI_COMM_NULL (-1)
#define MPI_SUCCESS 0
#define MPI_IDENT 0
#define MPI_MAX_PROCESSOR_NAME 256
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
#define MPI_IN_PLACE ((void*)1)
enum { MPI_CHAR = 1, MPI_SIGNED_CHAR, MPI_UNSIGNED_CHAR, MPI_BYTE, MPI_SHORT, MPI_UNSIGNED_SHORT,
       MPI_INT, MPI_UNSIGNED, MPI_LONG, MPI_UNSIGNED_LONG, MPI_LONG_LONG, MPI_LONG_LONG_INT,
       MPI_UNSIGNED_LONG_LONG, MPI_FLOAT, MPI_DOUBLE, MPI_LONG_DOUBLE, MPI_DOUBLE_INT,
       MPI_2INT, MPI_INT64_T, MPI_UINT64_T, MPI_DATATYPE_NULL };
enum { MPI_SUM = 1, MPI_MAX, MPI_MIN, MPI_MINLOC, MPI_MAXLOC, MPI_PROD, MPI_LOR, MPI_LAND, MPI_BOR, MPI_BAND };

static inline int oracle_mpi_type_size(MPI_Datatype t) {
   switch (t) {
   case MPI_CHAR: case MPI_SIGNED_CHAR: case MPI_UNSIGNED_CHAR: case MPI_BYTE: return 1;
   case MPI_SHORT: case MPI_UNSIGNED_SHORT: return 2;
   case MPI_INT: case MPI_UNSIGNED: case MPI_FLOAT: return 4;
   case MPI_LONG_DOUBLE: return sizeof(long double);
   case MPI_DOUBLE_INT: return 16;
   case MPI_2INT: return 8;
   default: return 8;
   }
}
static inline int MPI_Init(int* a, char*** b) { (void)a; (void)b; return 0; }
static inline int MPI_Initialized(int* f) { *f = 1; return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_rank(MPI_Comm c, int* r) { (void)c; *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm c, int* s) { (void)c; *s = 1; return 0; }
static inline int MPI_Comm_compare(MPI_Comm a, MPI_Comm b, int* r) { (void)a; (void)b; *r = MPI_IDENT; return 0; }
static inline int MPI_Comm_split(MPI_Comm c, int col, int key, MPI_Comm* n) { (void)col; (void)key; *n = c; return 0; }
static inline int MPI_Comm_dup(MPI_Comm c, MPI_Comm* n) { *n = c; return 0; }
static inline int MPI_Comm_free(MPI_Comm* c) { (void)c; return 0; }
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }
static inline int MPI_Abort(MPI_Comm c, int e) { (void)c; __builtin_exit(e); return 0; }
static inline double MPI_Wtime(void) { return 0.0; }
static inline int MPI_Get_processor_name(char* n, int* l) { strcpy(n, "oracle"); *l = 6; return 0; }
static inline int MPI_Bcast(void* b, int n, MPI_Datatype t, int root, MPI_Comm c) { (void)b; (void)n; (void)t; (void)root; (void)c; return 0; }
static inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op o, MPI_Comm c) {
   (void)o; (void)c; if (s != MPI_IN_PLACE && s != r) memcpy(r, s, (size_t)n * oracle_mpi_type_size(t)); return 0; }
static inline int MPI_Reduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op o, int root, MPI_Comm c) {
   (void)o; (void)root; (void)c; if (s != MPI_IN_PLACE && s != r && r) memcpy(r, s, (size_t)n * oracle_mpi_type_size(t)); return 0; }
static inline int MPI_Scan(const void* s, void* r, int n, MPI_Datatype t, MPI_Op o, MPI_Comm c) {
   (void)o; (void)c; memcpy(r, s, (size_t)n * oracle_mpi_type_size(t)); return 0; }
static inline int MPI_Exscan(const void* s, void* r, int n, MPI_Datatype t, MPI_Op o, MPI_Comm c) {
   (void)s; (void)o; (void)c; memset(r, 0, (size_t)n * oracle_mpi_type_size(t)); return 0; }
static inline int MPI_Gather(const void* s, int sn, MPI_Datatype st, void* r, int rn, MPI_Datatype rt, int root, MPI_Comm c) {
   (void)rn; (void)rt; (void)root; (void)c; if (r && s != r) memcpy(r, s, (size_t)sn * oracle_mpi_type_size(st)); return 0; }
static inline int MPI_Allgather(const void* s, int sn, MPI_Datatype st, void* r, int rn, MPI_Datatype rt, MPI_Comm c) {
   (void)rn; (void)rt; (void)c; if (s != MPI_IN_PLACE && s != r) memcpy(r, s, (size_t)sn * oracle_mpi_type_size(st)); return 0; }
static inline int MPI_Gatherv(const void* s, int sn, MPI_Datatype st, void* r, const int* rc, const int* d, MPI_Datatype rt, int root, MPI_Comm c) {
   (void)rc; (void)rt; (void)root; (void)c; if (r) memcpy((char*)r + (size_t)d[0] * oracle_mpi_type_size(st), s, (size_t)sn * oracle_mpi_type_size(st)); return 0; }
static inline int MPI_Allgatherv(const void* s, int sn, MPI_Datatype st, void* r, const int* rc, const int* d, MPI_Datatype rt, MPI_Comm c) {
   return MPI_Gatherv(s, sn, st, r, rc, d, rt, 0, c); }
static inline int MPI_Reduce_scatter(const void* s, void* r, const int* rc, MPI_Datatype t, MPI_Op o, MPI_Comm c) {
   (void)o; (void)c; memcpy(r, s, (size_t)rc[0] * oracle_mpi_type_size(t)); return 0; }
static inline int MPI_Send(const void* b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c) { (void)b; (void)n; (void)t; (void)d; (void)tag; (void)c; return 0; }
static inline int MPI_Recv(void* b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Status* st) { (void)b; (void)n; (void)t; (void)s; (void)tag; (void)c; (void)st; return 0; }
/* one rank: no message is ever pending */
static inline int MPI_Iprobe(int s, int tag, MPI_Comm c, int* flag, MPI_Status* st) { (void)s; (void)tag; (void)c; (void)st; *flag = 0; return 0; }
static inline int MPI_Isend(const void* b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c, MPI_Request* q) { (void)b; (void)n; (void)t; (void)d; (void)tag; (void)c; *q = 0; return 0; }
static inline int MPI_Irecv(void* b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Request* q) { (void)b; (void)n; (void)t; (void)s; (void)tag; (void)c; *q = 0; return 0; }
static inline int MPI_Wait(MPI_Request* q, MPI_Status* s) { (void)q; (void)s; return 0; }
static inline int MPI_Waitall(int n, MPI_Request* q, MPI_Status* s) { (void)n; (void)q; (void)s; return 0; }
static inline int MPI_Get_count(const MPI_Status* s, MPI_Datatype t, int* n) { (void)s; (void)t; *n = 0; return 0; }
static inline int MPI_Address(void* l, MPI_Aint* a) { *a = (MPI_Aint)l; return 0; }
static inline int MPI_Get_address(const void* l, MPI_Aint* a) { *a = (MPI_Aint)l; return 0; }
static inline int MPI_Type_commit(MPI_Datatype* t) { (void)t; return 0; }
static inline int MPI_Type_free(MPI_Datatype* t) { (void)t; return 0; }
static inline int MPI_Type_struct(int c, int* b, MPI_Aint* d, MPI_Datatype* t, MPI_Datatype* n) { (void)c; (void)b; (void)d; (void)t; *n = MPI_BYTE; return 0; }
static inline int MPI_Type_create_struct(int c, const int* b, const MPI_Aint* d, const MPI_Datatype* t, MPI_Datatype* n) { (void)c; (void)b; (void)d; (void)t; *n = MPI_BYTE; return 0; }
static inline int MPI_Type_contiguous(int c, MPI_Datatype o, MPI_Datatype* n) { (void)c; (void)o; *n = MPI_BYTE; return 0; }
#ifdef __cplusplus
}
#endif
#endif
