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
  int64_t node;   /* the node whose blocks are the work units */
  int64_t off;    /* byte offset of `node` inside one object */
  int64_t extent; /* extent of one object */
  int64_t per;    /* units per object (blocks of `node`, or 1) */
  int64_t u0, u1; /* this job's units [u0, u1) */
} job;

static void *run_job(void *p) {
  job *jb = (job *)p;
  walker *w = &jb->w;
  const onode *t = &w->nodes[jb->node];
  for (int64_t u = jb->u0; u < jb->u1; ++u) {
    const int64_t i = u / jb->per, j = u % jb->per;
    const int64_t base = i * jb->extent + jb->off;
    if (jb->per > 1)
      walk_run(w, t->child, base + j * t->stride, t->bl,
               w->nodes[t->child].extent);
    else
      walk(w, jb->node, base);
  }
  flush(w);
  return 0;
}

/* Pack (unpack=0) or unpack (unpack=1) `incount` objects of node `root`.
   `typed` is the typed buffer, `packed` the contiguous one.  Returns the
   number of packed bytes.

   With nthreads > 1 the work is split into units that each own one
   contiguous range of the packed buffer: the blocks of the outermost strided
   vector, found by stepping through one-block wrappers (a subarray's start
   displacement, a resized bound, a count-1 vector), times the objects.
   Each POSIX thread takes an even share of the units.  Without such a
   vector the units are whole objects. */
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

  int64_t node = root, off = 0, per = 1;
  for (;;) {
    const onode *n = &nodes[node];
    if (n->dense)
      break;
    if (n->kind == O_HIND && n->count == 1 && bls[n->aux] == 1) {
      off += displs[n->aux];
      node = n->child;
    } else if (n->kind == O_HVEC && n->count == 1 && n->bl == 1) {
      node = n->child;
    } else {
      break;
    }
  }
  const onode *s = &nodes[node];
  if (!s->dense && s->kind == O_HVEC && s->count > 1 &&
      s->count * s->bl * nodes[s->child].size == t->size)
    per = s->count;
  else {
    node = root;
    off = 0;
  }
  const int64_t units = incount * per;
  const int64_t unit_bytes = t->size / per;
  int64_t parts = nthreads < units ? nthreads : units;

  job jobs[256];
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
    jb->node = node;
    jb->off = off;
    jb->extent = t->extent;
    jb->per = per;
    jb->u0 = units * p / parts;
    jb->u1 = units * (p + 1) / parts;
    jb->w.pos = jb->u0 * unit_bytes;
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
