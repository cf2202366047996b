/*
 * Single-rank MPI shim — TEST INFRASTRUCTURE ONLY (part of the oracle).
 * See mpi.h for the contract.  Every derived datatype is reduced to a list of
 * (byte offset, byte length) segments inside one extent; pack, unpack and the
 * MPI-IO file view are all written in terms of that list.
 */
#include "mpi.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

shim_type shim_type_double = {0, sizeof(double), sizeof(double), 1, NULL, 0, {0}, {0}, {0}, 1};
shim_type shim_type_int = {0, sizeof(int), sizeof(int), 1, NULL, 0, {0}, {0}, {0}, 1};
shim_type shim_type_char = {0, 1, 1, 1, NULL, 0, {0}, {0}, {0}, 1};

static void shim_die(const char *what) {
  fprintf(stderr, "mpi_shim: %s\n", what);
  fflush(stderr);
  exit(97);
}

/* ---------------------------------------------------------------- segments */
typedef struct { size_t off, len; } seg_t;
typedef struct { seg_t *v; size_t n, cap; } seglist;

static void seg_push(seglist *s, size_t off, size_t len) {
  if (len == 0) return;
  if (s->n && s->v[s->n - 1].off + s->v[s->n - 1].len == off) {
    s->v[s->n - 1].len += len;
    return;
  }
  if (s->n == s->cap) {
    s->cap = s->cap ? 2 * s->cap : 64;
    s->v = (seg_t *)realloc(s->v, s->cap * sizeof(seg_t));
    if (!s->v) shim_die("out of memory");
  }
  s->v[s->n].off = off;
  s->v[s->n].len = len;
  s->n++;
}

static void seg_emit(const shim_type *t, size_t base, seglist *s) {
  if (t->kind == 0) {
    seg_push(s, base, t->size);
  } else if (t->kind == 1) {
    for (int c = 0; c < t->count; c++) seg_emit(t->base, base + (size_t)c * t->base->extent, s);
  } else {
    /* C-order subarray over t->base, up to 4 dims */
    int nd = t->ndims;
    int idx[4] = {0, 0, 0, 0};
    size_t stride[4];
    stride[nd - 1] = t->base->extent;
    for (int d = nd - 2; d >= 0; d--) stride[d] = stride[d + 1] * (size_t)t->sizes[d + 1];
    for (;;) {
      size_t off = base;
      for (int d = 0; d < nd; d++) off += (size_t)(t->starts[d] + idx[d]) * stride[d];
      seg_emit(t->base, off, s);
      int d = nd - 1;
      while (d >= 0) {
        if (++idx[d] < t->subsizes[d]) break;
        idx[d] = 0;
        d--;
      }
      if (d < 0) break;
    }
  }
}

static seglist type_segments(const shim_type *t) {
  seglist s = {NULL, 0, 0};
  seg_emit(t, 0, &s);
  return s;
}

static void pack(const void *buf, int count, const shim_type *t, char *out) {
  seglist s = type_segments(t);
  const char *b = (const char *)buf;
  for (int c = 0; c < count; c++)
    for (size_t i = 0; i < s.n; i++) {
      memcpy(out, b + (size_t)c * t->extent + s.v[i].off, s.v[i].len);
      out += s.v[i].len;
    }
  free(s.v);
}

static void unpack(const char *in, void *buf, int count, const shim_type *t) {
  seglist s = type_segments(t);
  char *b = (char *)buf;
  for (int c = 0; c < count; c++)
    for (size_t i = 0; i < s.n; i++) {
      memcpy(b + (size_t)c * t->extent + s.v[i].off, in, s.v[i].len);
      in += s.v[i].len;
    }
  free(s.v);
}

/* ------------------------------------------------------------ environment */
int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Abort(MPI_Comm comm, int code) {
  (void)comm;
  fprintf(stderr, "MPI_Abort(%d)\n", code);
  fflush(stderr);
  exit(code ? code : 1);
}
int MPI_Barrier(MPI_Comm comm) { (void)comm; return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm comm, int *size) { (void)comm; *size = 1; return MPI_SUCCESS; }
int MPI_Comm_rank(MPI_Comm comm, int *rank) { (void)comm; *rank = 0; return MPI_SUCCESS; }
int MPI_Comm_set_errhandler(MPI_Comm comm, MPI_Errhandler h) { (void)comm; (void)h; return MPI_SUCCESS; }
int MPI_Get_processor_name(char *name, int *len) {
  strcpy(name, "oracle-shim");
  *len = (int)strlen(name);
  return MPI_SUCCESS;
}
double MPI_Wtime(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
int MPI_Error_class(int code, int *cls) { *cls = code; return MPI_SUCCESS; }
int MPI_Error_string(int code, char *str, int *len) {
  snprintf(str, MPI_MAX_ERROR_STRING, "mpi_shim error %d", code);
  *len = (int)strlen(str);
  return MPI_SUCCESS;
}

int MPI_Cart_create(MPI_Comm old, int ndims, const int *dims, const int *periods, int reorder,
                    MPI_Comm *cart) {
  (void)old; (void)periods; (void)reorder;
  for (int d = 0; d < ndims; d++)
    if (dims[d] != 1) shim_die("Cartesian topology must be 1x1 (XDIM = YDIM = 1)");
  *cart = 1;
  return MPI_SUCCESS;
}
int MPI_Cart_coords(MPI_Comm comm, int rank, int maxdims, int *coords) {
  (void)comm; (void)rank;
  for (int d = 0; d < maxdims; d++) coords[d] = 0;
  return MPI_SUCCESS;
}
int MPI_Cart_rank(MPI_Comm comm, const int *coords, int *rank) {
  (void)comm; (void)coords;
  *rank = 0;
  return MPI_SUCCESS;
}

/* -------------------------------------------------------------- datatypes */
int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype *newtype) {
  shim_type *t = (shim_type *)calloc(1, sizeof(shim_type));
  t->kind = 1;
  t->count = count;
  t->base = old;
  t->size = (size_t)count * old->size;
  t->extent = (size_t)count * old->extent;
  *newtype = t;
  return MPI_SUCCESS;
}
int MPI_Type_create_subarray(int ndims, const int *sizes, const int *subsizes, const int *starts,
                             int order, MPI_Datatype old, MPI_Datatype *newtype) {
  if (order != MPI_ORDER_C) shim_die("only MPI_ORDER_C subarrays are supported");
  if (ndims < 1 || ndims > 4) shim_die("subarray rank out of range");
  shim_type *t = (shim_type *)calloc(1, sizeof(shim_type));
  t->kind = 2;
  t->base = old;
  t->ndims = ndims;
  size_t n = 1, full = 1;
  for (int d = 0; d < ndims; d++) {
    if (starts[d] < 0 || subsizes[d] < 0 || starts[d] + subsizes[d] > sizes[d])
      shim_die("subarray out of bounds");
    t->sizes[d] = sizes[d];
    t->subsizes[d] = subsizes[d];
    t->starts[d] = starts[d];
    n *= (size_t)subsizes[d];
    full *= (size_t)sizes[d];
  }
  t->size = n * old->size;
  t->extent = full * old->extent;
  *newtype = t;
  return MPI_SUCCESS;
}
int MPI_Type_commit(MPI_Datatype *t) { (*t)->committed = 1; return MPI_SUCCESS; }
int MPI_Type_free(MPI_Datatype *t) {
  /* element types may be shared by several derived types; leak them (tiny) */
  *t = NULL;
  return MPI_SUCCESS;
}

/* ----------------------------------------------------- point to point */
struct shim_req {
  int is_send;
  void *buf;
  int count;
  MPI_Datatype type;
  int tag;
};

typedef struct pending {
  int tag;
  struct shim_req *req; /* receive waiting for a send */
  char *data;           /* send waiting for a receive (packed copy) */
  size_t bytes;
  struct pending *next;
} pending;

static pending *q_sends = NULL, *q_recvs = NULL;

static void q_append(pending **q, pending *p) {
  p->next = NULL;
  while (*q) q = &(*q)->next;
  *q = p;
}
static pending *q_take(pending **q, int tag) {
  for (; *q; q = &(*q)->next)
    if ((*q)->tag == tag) {
      pending *p = *q;
      *q = p->next;
      return p;
    }
  return NULL;
}

int MPI_Send_init(const void *buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm comm,
                  MPI_Request *req) {
  (void)dest; (void)comm;
  struct shim_req *r = (struct shim_req *)calloc(1, sizeof(*r));
  r->is_send = 1;
  r->buf = (void *)buf;
  r->count = count;
  r->type = t;
  r->tag = tag;
  *req = r;
  return MPI_SUCCESS;
}
int MPI_Recv_init(void *buf, int count, MPI_Datatype t, int source, int tag, MPI_Comm comm,
                  MPI_Request *req) {
  (void)source; (void)comm;
  struct shim_req *r = (struct shim_req *)calloc(1, sizeof(*r));
  r->is_send = 0;
  r->buf = buf;
  r->count = count;
  r->type = t;
  r->tag = tag;
  *req = r;
  return MPI_SUCCESS;
}

static void deliver(const char *data, size_t bytes, struct shim_req *recv) {
  size_t want = (size_t)recv->count * recv->type->size;
  if (bytes > want) shim_die("message truncated (send larger than receive)");
  unpack(data, recv->buf, recv->count, recv->type);
}

int MPI_Startall(int n, MPI_Request *reqs) {
  for (int i = 0; i < n; i++) {
    struct shim_req *r = reqs[i];
    if (!r) continue;
    if (r->is_send) {
      size_t bytes = (size_t)r->count * r->type->size;
      pending *w = q_take(&q_recvs, r->tag);
      char *tmp = (char *)malloc(bytes ? bytes : 1);
      pack(r->buf, r->count, r->type, tmp);
      if (w) {
        deliver(tmp, bytes, w->req);
        free(tmp);
        free(w);
      } else {
        pending *p = (pending *)calloc(1, sizeof(*p));
        p->tag = r->tag;
        p->data = tmp;
        p->bytes = bytes;
        q_append(&q_sends, p);
      }
    } else {
      pending *s = q_take(&q_sends, r->tag);
      if (s) {
        deliver(s->data, s->bytes, r);
        free(s->data);
        free(s);
      } else {
        pending *p = (pending *)calloc(1, sizeof(*p));
        p->tag = r->tag;
        p->req = r;
        q_append(&q_recvs, p);
      }
    }
  }
  if (q_sends || q_recvs) shim_die("unmatched persistent request after MPI_Startall");
  return MPI_SUCCESS;
}
int MPI_Testall(int n, MPI_Request *reqs, int *flag, MPI_Status *st) {
  (void)n; (void)reqs; (void)st;
  *flag = 1;
  return MPI_SUCCESS;
}
int MPI_Waitall(int n, MPI_Request *reqs, MPI_Status *st) { (void)n; (void)reqs; (void)st; return MPI_SUCCESS; }
int MPI_Request_free(MPI_Request *req) {
  free(*req);
  *req = MPI_REQUEST_NULL;
  return MPI_SUCCESS;
}

int MPI_Sendrecv(const void *sbuf, int scount, MPI_Datatype stype, int dest, int stag, void *rbuf,
                 int rcount, MPI_Datatype rtype, int source, int rtag, MPI_Comm comm,
                 MPI_Status *st) {
  (void)dest; (void)source; (void)comm;
  if (stag != rtag) shim_die("self Sendrecv with mismatched tags");
  size_t bytes = (size_t)scount * stype->size;
  if (bytes != (size_t)rcount * rtype->size) shim_die("self Sendrecv with mismatched sizes");
  char *tmp = (char *)malloc(bytes ? bytes : 1);
  pack(sbuf, scount, stype, tmp);
  unpack(tmp, rbuf, rcount, rtype);
  free(tmp);
  if (st) {
    st->count_bytes = (long long)bytes;
    st->MPI_SOURCE = 0;
    st->MPI_TAG = rtag;
    st->MPI_ERROR = 0;
  }
  return MPI_SUCCESS;
}

int MPI_Reduce(const void *sbuf, void *rbuf, int count, MPI_Datatype t, MPI_Op op, int root, MPI_Comm comm) {
  (void)op; (void)root; (void)comm;
  memmove(rbuf, sbuf, (size_t)count * t->size);
  return MPI_SUCCESS;
}
int MPI_Allreduce(const void *sbuf, void *rbuf, int count, MPI_Datatype t, MPI_Op op, MPI_Comm comm) {
  (void)op; (void)comm;
  memmove(rbuf, sbuf, (size_t)count * t->size);
  return MPI_SUCCESS;
}
int MPI_Bcast(void *buf, int count, MPI_Datatype t, int root, MPI_Comm comm) {
  (void)buf; (void)count; (void)t; (void)root; (void)comm;
  return MPI_SUCCESS;
}
int MPI_Get_count(const MPI_Status *st, MPI_Datatype t, int *count) {
  *count = (int)(st->count_bytes / (long long)t->size);
  return MPI_SUCCESS;
}

int MPI_Info_create(MPI_Info *info) { *info = 0; return MPI_SUCCESS; }
int MPI_Info_set(MPI_Info info, const char *key, const char *value) { (void)info; (void)key; (void)value; return MPI_SUCCESS; }
int MPI_Info_free(MPI_Info *info) { *info = 0; return MPI_SUCCESS; }

/* ------------------------------------------------------------------ MPI-IO */
struct shim_file {
  FILE *fp;
  MPI_Offset disp;
  MPI_Datatype etype, filetype;
  size_t pos; /* individual file pointer: bytes of the view's data stream consumed */
};

int MPI_File_open(MPI_Comm comm, const char *name, int amode, MPI_Info info, MPI_File *fh) {
  (void)comm; (void)info;
  FILE *fp;
  if (amode & MPI_MODE_RDONLY) {
    fp = fopen(name, "rb");
  } else {
    fp = fopen(name, "r+b");
    if (!fp && (amode & MPI_MODE_CREATE)) fp = fopen(name, "w+b");
  }
  if (!fp) {
    fprintf(stderr, "mpi_shim: cannot open %s\n", name);
    exit(98);
  }
  struct shim_file *f = (struct shim_file *)calloc(1, sizeof(*f));
  f->fp = fp;
  f->disp = 0;
  f->etype = MPI_CHAR;
  f->filetype = MPI_CHAR;
  f->pos = 0;
  *fh = f;
  return MPI_SUCCESS;
}
int MPI_File_set_view(MPI_File fh, MPI_Offset disp, MPI_Datatype etype, MPI_Datatype filetype,
                      const char *rep, MPI_Info info) {
  (void)rep; (void)info;
  fh->disp = disp;
  fh->etype = etype;
  fh->filetype = filetype;
  fh->pos = 0;
  return MPI_SUCCESS;
}

/* walk the data stream through the tiled filetype from stream byte `start`,
   reading or writing `bytes` */
static int file_stream_at(MPI_File fh, char *data, size_t bytes, int writing, size_t start) {
  seglist s = type_segments(fh->filetype);
  size_t done = 0, skip = start;
  for (size_t tile = 0; done < bytes; tile++) {
    for (size_t i = 0; i < s.n && done < bytes; i++) {
      size_t seg_off = s.v[i].off, len = s.v[i].len;
      if (skip >= len) {
        skip -= len;
        continue;
      }
      seg_off += skip;
      len -= skip;
      skip = 0;
      if (len > bytes - done) len = bytes - done;
      long long off = fh->disp + (long long)(tile * fh->filetype->extent + seg_off);
      if (fseeko(fh->fp, (off_t)off, SEEK_SET) != 0) { free(s.v); return -1; }
      size_t got = writing ? fwrite(data + done, 1, len, fh->fp) : fread(data + done, 1, len, fh->fp);
      if (got != len) { free(s.v); return -1; }
      done += len;
    }
    if (s.n == 0) break;
  }
  free(s.v);
  return 0;
}
static int file_stream(MPI_File fh, char *data, size_t bytes, int writing) {
  return file_stream_at(fh, data, bytes, writing, 0);
}

/* independent read at the individual file pointer, which it advances */
int MPI_File_read(MPI_File fh, void *buf, int count, MPI_Datatype t, MPI_Status *st) {
  size_t bytes = (size_t)count * t->size;
  char *tmp = (char *)malloc(bytes ? bytes : 1);
  if (file_stream_at(fh, tmp, bytes, 0, fh->pos) != 0) shim_die("short read in MPI_File_read");
  fh->pos += bytes;
  unpack(tmp, buf, count, t);
  free(tmp);
  if (st) st->count_bytes = (long long)bytes;
  return MPI_SUCCESS;
}
/* collective read at an explicit offset in etype units of the view */
int MPI_File_read_at_all(MPI_File fh, MPI_Offset offset, void *buf, int count, MPI_Datatype t, MPI_Status *st) {
  size_t bytes = (size_t)count * t->size;
  char *tmp = (char *)malloc(bytes ? bytes : 1);
  if (file_stream_at(fh, tmp, bytes, 0, (size_t)offset * fh->etype->size) != 0)
    shim_die("short read in MPI_File_read_at_all");
  unpack(tmp, buf, count, t);
  free(tmp);
  if (st) st->count_bytes = (long long)bytes;
  return MPI_SUCCESS;
}

int MPI_File_read_all(MPI_File fh, void *buf, int count, MPI_Datatype t, MPI_Status *st) {
  size_t bytes = (size_t)count * t->size;
  char *tmp = (char *)malloc(bytes ? bytes : 1);
  if (file_stream(fh, tmp, bytes, 0) != 0) shim_die("short read in MPI_File_read_all");
  unpack(tmp, buf, count, t);
  free(tmp);
  if (st) st->count_bytes = (long long)bytes;
  return MPI_SUCCESS;
}
int MPI_File_write_all(MPI_File fh, const void *buf, int count, MPI_Datatype t, MPI_Status *st) {
  size_t bytes = (size_t)count * t->size;
  char *tmp = (char *)malloc(bytes ? bytes : 1);
  pack(buf, count, t, tmp);
  if (file_stream(fh, tmp, bytes, 1) != 0) shim_die("short write in MPI_File_write_all");
  free(tmp);
  if (st) st->count_bytes = (long long)bytes;
  return MPI_SUCCESS;
}
int MPI_File_close(MPI_File *fh) {
  if (*fh) {
    fclose((*fh)->fp);
    free(*fh);
  }
  *fh = NULL;
  return MPI_SUCCESS;
}
