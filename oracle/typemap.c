/* ORACLE -- test infrastructure only.  Nothing in the product links this.

   CPU type-map walker for MPI_Pack / MPI_Unpack, written from the MPI-3.1
   type-map definitions (section 4.1.2 Datatype constructors, 4.2 Pack/Unpack).
   It stands in for "the underlying MPI library's own MPI_Pack" which the
   reference compares against (test/pack_unpack.cpp:62-68, 90-97) but which is
   absent on this machine.  It is also the timed CPU baseline (the reference's
   host path hands host buffers to the library's MPI_Pack, src/pack.cpp:51-55).

   Types arrive as a node array built by oracle/oracle.py.  Every constructor
   is lowered there to one of four node kinds:
     NAMED   : `size` contiguous bytes
     HVEC    : `count` blocks at byte stride `stride`, each block `bl`
               copies of `child` at the child's extent
     HIND    : `count` blocks, block i = bls[i] copies of `child` at byte
               displacement displs[i]
     STRUCT  : block i = bls[i] copies of child kinds[i] at displs[i]
               (children listed in the `kids` array)
   A node whose type map is one ascending contiguous run carries dense=1 and
   is copied as one run.  Runs that are adjacent in the source are merged.
*/
#include <pthread.h>
#include <stdint.h>
#include <string.h>

enum { O_NAMED = 0, O_HVEC = 1, O_HIND = 2, O_STRUCT = 3 };

typedef struct {
  int32_t kind;
  int32_t dense;
  int64_t child;  /* HVEC/HIND: child node */
  int64_t count;  /* blocks */
  int64_t bl;     /* HVEC: copies per block */
  int64_t stride; /* HVEC: bytes between blocks */
  int64_t size;   /* packed bytes of one instance */
  int64_t lb;     /* lower bound */
  int64_t extent; /* ub - lb */
  int64_t aux;    /* HIND/STRUCT: first index into bls/displs/kids */
} onode;

typedef struct {
  const onode *nodes;
  const int64_t *bls, *displs, *kids;
  const char *in;
  char *out;
  int64_t pos;
  int64_t roff, rlen; /* pending merged run (source offsets) */
  int unpack;
} walker;

static void flush(walker *w) {
  if (w->rlen <= 0)
    return;
  if (w->unpack)
    memcpy((char *)w->in + w->roff, w->out + w->pos, (size_t)w->rlen);
  else
    memcpy(w->out + w->pos, w->in + w->roff, (size_t)w->rlen);
  w->pos += w->rlen;
  w->rlen = 0;
}

static void emit(walker *w, int64_t off, int64_t len) {
  if (len <= 0)
    return;
  if (w->rlen > 0 && off == w->roff + w->rlen) {
    w->rlen += len;
    return;
  }
  flush(w);
  w->roff = off;
  w->rlen = len;
}

static void walk(walker *w, int64_t n, int64_t base);

/* `cnt` copies of node c, copy k at base + k*step */
static void walk_run(walker *w, int64_t c, int64_t base, int64_t cnt,
                     int64_t step) {
  const onode *nc = &w->nodes[c];
  if (nc->dense && step == nc->size) {
    emit(w, base + nc->lb, cnt * nc->size);
    return;
  }
  for (int64_t k = 0; k < cnt; ++k)
    walk(w, c, base + k * step);
}

static void walk(walker *w, int64_t n, int64_t base) {
  const onode *t = &w->nodes[n];
  if (t->dense) {
    emit(w, base + t->lb, t->size);
    return;
  }
  switch (t->kind) {
  case O_NAMED:
    emit(w, base, t->size);
    return;
  case O_HVEC:
    for (int64_t j = 0; j < t->count; ++j)
      walk_run(w, t->child, base + j * t->stride, t->bl,
               w->nodes[t->child].extent);
    return;
  case O_HIND:
    for (int64_t i = 0; i < t->count; ++i)
      walk_run(w, t->child, base + w->displs[t->aux + i], w->bls[t->aux + i],
               w->nodes[t->child].extent);
    return;
  case O_STRUCT:
    for (int64_t i = 0; i < t->count; ++i) {
      int64_t c = w->kids[t->aux + i];
      walk_run(w, c, base + w->displs[t->aux + i], w->bls[t->aux + i],
               w->nodes[c].extent);
    }
    return;
  }
}

typedef struct {
  walker w;
  int64_t root, obj0, obj1; /* objects [obj0, obj1) */
  int64_t j0, j1;           /* or, with one object, root blocks [j0, j1) */
  int64_t extent;
} job;

static void *run_job(void *p) {
  job *jb = (job *)p;
  walker *w = &jb->w;
  if (jb->j1 > jb->j0) {
    const onode *t = &w->nodes[jb->root];
    for (int64_t j = jb->j0; j < jb->j1; ++j)
      walk_run(w, t->child, j * t->stride, t->bl, w->nodes[t->child].extent);
  } else {
    for (int64_t i = jb->obj0; i < jb->obj1; ++i)
      walk(w, jb->root, i * jb->extent);
  }
  flush(w);
  return 0;
}

/* Pack (unpack=0) or unpack (unpack=1) `incount` objects of node `root`.
   `typed` is the typed buffer, `packed` the contiguous one.  Returns the
   number of packed bytes.  With nthreads > 1 the objects (or, for a single
   HVEC object, its blocks) are split evenly across POSIX threads. */
int64_t oracle_walk(const onode *nodes, int64_t root, const int64_t *bls,
                    const int64_t *displs, const int64_t *kids, char *typed,
                    int64_t incount, char *packed, int unpack, int nthreads) {
  const onode *t = &nodes[root];
  const int64_t total = incount * t->size;
  if (total == 0)
    return 0;
  if (nthreads < 1)
    nthreads = 1;
  if (nthreads > 256)
    nthreads = 256;
  job jobs[256];
  int64_t parts = 1, by_blocks = 0;
  if (nthreads > 1 && incount >= nthreads) {
    parts = nthreads;
  } else if (nthreads > 1 && incount == 1 && t->kind == O_HVEC && !t->dense &&
             t->count >= nthreads) {
    parts = nthreads;
    by_blocks = 1;
  }
  const int64_t per_block = t->bl * nodes[t->child].size;
  for (int64_t p = 0; p < parts; ++p) {
    job *jb = &jobs[p];
    memset(jb, 0, sizeof(*jb));
    jb->w.nodes = nodes;
    jb->w.bls = bls;
    jb->w.displs = displs;
    jb->w.kids = kids;
    jb->w.in = typed;
    jb->w.out = packed;
    jb->w.unpack = unpack;
    jb->root = root;
    jb->extent = t->extent;
    if (by_blocks) {
      jb->j0 = t->count * p / parts;
      jb->j1 = t->count * (p + 1) / parts;
      jb->w.pos = jb->j0 * per_block;
    } else {
      jb->obj0 = incount * p / parts;
      jb->obj1 = incount * (p + 1) / parts;
      jb->w.pos = jb->obj0 * t->size;
    }
  }
  if (parts == 1) {
    run_job(&jobs[0]);
    return jobs[0].w.pos;
  }
  pthread_t th[256];
  for (int64_t p = 1; p < parts; ++p)
    pthread_create(&th[p], 0, run_job, &jobs[p]);
  run_job(&jobs[0]);
  for (int64_t p = 1; p < parts; ++p)
    pthread_join(th[p], 0);
  return total;
}
