/* Flat-file stand-in for the HDF5 subset used by the reference (see hdf5.h).
 * Test infrastructure only. */
#include "hdf5.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define MAX_OBJ 4096
#define MAX_DSET 256

typedef struct {
  char name[128];
  int type; /* 0 double, 1 int32 */
  int ndims;
  hsize_t dims[8];
  char *data;
  size_t nbytes;
} dset_t;

typedef struct {
  char path[512];
  int writable;
  int discard;
  int ndset;
  dset_t dset[MAX_DSET];
} file_t;

typedef struct {
  int ndims;
  hsize_t dims[8];
  int has_sel;
  hsize_t start[8], count[8];
} space_t;

enum { OBJ_FREE = 0, OBJ_FILE, OBJ_SPACE, OBJ_DSET, OBJ_PLIST };
typedef struct {
  int kind;
  void *ptr;     /* file_t* or space_t* */
  int dset_idx;  /* for OBJ_DSET */
  hid_t file;    /* for OBJ_DSET */
} obj_t;

static obj_t g_obj[MAX_OBJ];

static hid_t new_obj(int kind, void *ptr) {
  for (int i = 1; i < MAX_OBJ; i++) {
    if (g_obj[i].kind == OBJ_FREE) {
      g_obj[i].kind = kind;
      g_obj[i].ptr = ptr;
      return (hid_t)i;
    }
  }
  return -1;
}

static obj_t *get_obj(hid_t id, int kind) {
  if (id <= 0 || id >= MAX_OBJ) return NULL;
  if (g_obj[id].kind != kind) return NULL;
  return &g_obj[id];
}

static size_t type_size(int type) { return type == 0 ? 8 : 4; }
static int type_code(hid_t t) { return t == H5T_NATIVE_INT ? 1 : 0; }

static int env_discard(void) {
  const char *e = getenv("GOP_H5_DISCARD");
  return e && e[0] == '1';
}

static int load_file(file_t *f) {
  FILE *fp = fopen(f->path, "rb");
  if (!fp) return -1;
  char magic[8];
  if (fread(magic, 1, 8, fp) != 8 || memcmp(magic, "GOPRAW01", 8) != 0) {
    fclose(fp);
    return -1;
  }
  uint32_t n = 0;
  if (fread(&n, 4, 1, fp) != 1) {
    fclose(fp);
    return -1;
  }
  for (uint32_t r = 0; r < n && f->ndset < MAX_DSET; r++) {
    dset_t *d = &f->dset[f->ndset];
    uint32_t len = 0;
    int32_t type = 0, nd = 0;
    uint64_t nbytes = 0;
    if (fread(&len, 4, 1, fp) != 1 || len >= sizeof(d->name)) break;
    if (fread(d->name, 1, len, fp) != len) break;
    d->name[len] = 0;
    if (fread(&type, 4, 1, fp) != 1 || fread(&nd, 4, 1, fp) != 1) break;
    d->type = type;
    d->ndims = nd;
    for (int k = 0; k < nd; k++) {
      uint64_t v;
      if (fread(&v, 8, 1, fp) != 1) break;
      d->dims[k] = v;
    }
    if (fread(&nbytes, 8, 1, fp) != 1) break;
    d->data = (char *)malloc(nbytes ? nbytes : 1);
    d->nbytes = nbytes;
    if (fread(d->data, 1, nbytes, fp) != nbytes) break;
    f->ndset++;
  }
  fclose(fp);
  return 0;
}

static int save_file(file_t *f) {
  FILE *fp = fopen(f->path, "wb");
  if (!fp) return -1;
  fwrite("GOPRAW01", 1, 8, fp);
  uint32_t n = (uint32_t)f->ndset;
  fwrite(&n, 4, 1, fp);
  for (int r = 0; r < f->ndset; r++) {
    dset_t *d = &f->dset[r];
    uint32_t len = (uint32_t)strlen(d->name);
    int32_t type = d->type, nd = d->ndims;
    uint64_t nbytes = d->nbytes;
    fwrite(&len, 4, 1, fp);
    fwrite(d->name, 1, len, fp);
    fwrite(&type, 4, 1, fp);
    fwrite(&nd, 4, 1, fp);
    for (int k = 0; k < nd; k++) {
      uint64_t v = d->dims[k];
      fwrite(&v, 8, 1, fp);
    }
    fwrite(&nbytes, 8, 1, fp);
    fwrite(d->data, 1, d->nbytes, fp);
  }
  fclose(fp);
  return 0;
}

hid_t H5Fcreate(const char *name, unsigned flags, hid_t fcpl, hid_t fapl) {
  (void)flags;
  (void)fcpl;
  (void)fapl;
  file_t *f = (file_t *)calloc(1, sizeof(file_t));
  snprintf(f->path, sizeof(f->path), "%s", name);
  f->writable = 1;
  f->discard = env_discard();
  return new_obj(OBJ_FILE, f);
}

hid_t H5Fopen(const char *name, unsigned flags, hid_t fapl) {
  (void)fapl;
  file_t *f = (file_t *)calloc(1, sizeof(file_t));
  snprintf(f->path, sizeof(f->path), "%s", name);
  f->writable = (flags == H5F_ACC_RDWR);
  f->discard = f->writable && env_discard();
  if (!f->discard && load_file(f) != 0) {
    free(f);
    return -1;
  }
  return new_obj(OBJ_FILE, f);
}

herr_t H5Fclose(hid_t file) {
  obj_t *o = get_obj(file, OBJ_FILE);
  if (!o) return -1;
  file_t *f = (file_t *)o->ptr;
  int rc = 0;
  if (f->writable && !f->discard) rc = save_file(f);
  for (int r = 0; r < f->ndset; r++) free(f->dset[r].data);
  free(f);
  o->kind = OBJ_FREE;
  return rc;
}

hid_t H5Screate_simple(int rank, const hsize_t *dims, const hsize_t *maxdims) {
  (void)maxdims;
  if (rank < 1 || rank > 8) return -1;
  space_t *s = (space_t *)calloc(1, sizeof(space_t));
  s->ndims = rank;
  for (int k = 0; k < rank; k++) s->dims[k] = dims[k];
  return new_obj(OBJ_SPACE, s);
}

herr_t H5Sclose(hid_t space) {
  obj_t *o = get_obj(space, OBJ_SPACE);
  if (!o) return -1;
  free(o->ptr);
  o->kind = OBJ_FREE;
  return 0;
}

herr_t H5Sselect_hyperslab(hid_t space, H5S_seloper_t op, const hsize_t *start,
                           const hsize_t *stride, const hsize_t *count,
                           const hsize_t *block) {
  (void)op;
  if (stride || block) return -1;
  obj_t *o = get_obj(space, OBJ_SPACE);
  if (!o) return -1;
  space_t *s = (space_t *)o->ptr;
  for (int k = 0; k < s->ndims; k++) {
    if (start[k] + count[k] > s->dims[k]) return -1;
    s->start[k] = start[k];
    s->count[k] = count[k];
  }
  s->has_sel = 1;
  return 0;
}

int H5Sget_simple_extent_ndims(hid_t space) {
  obj_t *o = get_obj(space, OBJ_SPACE);
  if (!o) return -1;
  return ((space_t *)o->ptr)->ndims;
}

int H5Sget_simple_extent_dims(hid_t space, hsize_t *dims, hsize_t *maxdims) {
  obj_t *o = get_obj(space, OBJ_SPACE);
  if (!o) return -1;
  space_t *s = (space_t *)o->ptr;
  for (int k = 0; k < s->ndims; k++) {
    if (dims) dims[k] = s->dims[k];
    if (maxdims) maxdims[k] = s->dims[k];
  }
  return s->ndims;
}

hid_t H5Pcreate(hid_t cls) {
  (void)cls;
  return new_obj(OBJ_PLIST, NULL);
}
herr_t H5Pclose(hid_t plist) {
  obj_t *o = get_obj(plist, OBJ_PLIST);
  if (!o) return -1;
  o->kind = OBJ_FREE;
  return 0;
}
herr_t H5Pset_chunk(hid_t plist, int ndims, const hsize_t *dims) {
  (void)ndims;
  (void)dims;
  return get_obj(plist, OBJ_PLIST) ? 0 : -1;
}
herr_t H5Pset_deflate(hid_t plist, unsigned level) {
  (void)level;
  return get_obj(plist, OBJ_PLIST) ? 0 : -1;
}

hid_t H5Dcreate2(hid_t loc, const char *name, hid_t type, hid_t space,
                 hid_t lcpl, hid_t dcpl, hid_t dapl) {
  (void)lcpl;
  (void)dcpl;
  (void)dapl;
  obj_t *fo = get_obj(loc, OBJ_FILE);
  obj_t *so = get_obj(space, OBJ_SPACE);
  if (!fo || !so) return -1;
  file_t *f = (file_t *)fo->ptr;
  space_t *s = (space_t *)so->ptr;
  const char *nm = name[0] == '/' ? name + 1 : name;
  int idx = -1;
  for (int r = 0; r < f->ndset; r++)
    if (strcmp(f->dset[r].name, nm) == 0) return -1; /* exists */
  if (f->ndset >= MAX_DSET) return -1;
  idx = f->ndset++;
  dset_t *d = &f->dset[idx];
  snprintf(d->name, sizeof(d->name), "%s", nm);
  d->type = type_code(type);
  d->ndims = s->ndims;
  size_t n = 1;
  for (int k = 0; k < s->ndims; k++) {
    d->dims[k] = s->dims[k];
    n *= (size_t)s->dims[k];
  }
  d->nbytes = n * type_size(d->type);
  d->data = f->discard ? NULL : (char *)calloc(d->nbytes ? d->nbytes : 1, 1);
  hid_t id = new_obj(OBJ_DSET, NULL);
  if (id < 0) return -1;
  g_obj[id].dset_idx = idx;
  g_obj[id].file = loc;
  return id;
}

hid_t H5Dopen2(hid_t loc, const char *name, hid_t dapl) {
  (void)dapl;
  obj_t *fo = get_obj(loc, OBJ_FILE);
  if (!fo) return -1;
  file_t *f = (file_t *)fo->ptr;
  const char *nm = name[0] == '/' ? name + 1 : name;
  for (int r = 0; r < f->ndset; r++) {
    if (strcmp(f->dset[r].name, nm) == 0) {
      hid_t id = new_obj(OBJ_DSET, NULL);
      if (id < 0) return -1;
      g_obj[id].dset_idx = r;
      g_obj[id].file = loc;
      return id;
    }
  }
  return -1;
}

herr_t H5Dclose(hid_t dset) {
  obj_t *o = get_obj(dset, OBJ_DSET);
  if (!o) return -1;
  o->kind = OBJ_FREE;
  return 0;
}

static dset_t *dset_of(hid_t dset) {
  obj_t *o = get_obj(dset, OBJ_DSET);
  if (!o) return NULL;
  obj_t *fo = get_obj(o->file, OBJ_FILE);
  if (!fo) return NULL;
  return &((file_t *)fo->ptr)->dset[o->dset_idx];
}

static file_t *file_of(hid_t dset) {
  obj_t *o = get_obj(dset, OBJ_DSET);
  if (!o) return NULL;
  obj_t *fo = get_obj(o->file, OBJ_FILE);
  return fo ? (file_t *)fo->ptr : NULL;
}

hid_t H5Dget_space(hid_t dset) {
  dset_t *d = dset_of(dset);
  if (!d) return -1;
  return H5Screate_simple(d->ndims, d->dims, NULL);
}

/* Copy between the contiguous user buffer and the hyperslab of the dataset
 * selected in filespace (whole dataset when filespace is H5S_ALL). */
static herr_t transfer(hid_t dset, hid_t filespace, char *buf, int to_file) {
  dset_t *d = dset_of(dset);
  file_t *f = file_of(dset);
  if (!d || !f) return -1;
  if (f->discard) return 0;
  size_t es = type_size(d->type);
  hsize_t start[8] = {0}, count[8];
  for (int k = 0; k < d->ndims; k++) count[k] = d->dims[k];
  if (filespace != H5S_ALL) {
    obj_t *so = get_obj(filespace, OBJ_SPACE);
    if (!so) return -1;
    space_t *s = (space_t *)so->ptr;
    if (s->ndims != d->ndims) return -1;
    if (s->has_sel) {
      for (int k = 0; k < d->ndims; k++) {
        start[k] = s->start[k];
        count[k] = s->count[k];
      }
    }
  }
  /* rows along the last dimension are contiguous */
  int nd = d->ndims;
  size_t row = (size_t)count[nd - 1];
  size_t nrows = 1;
  for (int k = 0; k < nd - 1; k++) nrows *= (size_t)count[k];
  hsize_t idx[8] = {0};
  size_t pos = 0;
  for (size_t r = 0; r < nrows; r++) {
    size_t off = 0;
    for (int k = 0; k < nd; k++) {
      hsize_t c = (k < nd - 1 ? idx[k] : 0) + start[k];
      off = off * (size_t)d->dims[k] + (size_t)c;
    }
    if (to_file)
      memcpy(d->data + off * es, buf + pos * es, row * es);
    else
      memcpy(buf + pos * es, d->data + off * es, row * es);
    pos += row;
    for (int k = nd - 2; k >= 0; k--) {
      if (++idx[k] < count[k]) break;
      idx[k] = 0;
    }
  }
  return 0;
}

herr_t H5Dwrite(hid_t dset, hid_t memtype, hid_t memspace, hid_t filespace,
                hid_t plist, const void *buf) {
  (void)memtype;
  (void)memspace;
  (void)plist;
  return transfer(dset, filespace, (char *)buf, 1);
}

herr_t H5Dread(hid_t dset, hid_t memtype, hid_t memspace, hid_t filespace,
               hid_t plist, void *buf) {
  (void)memtype;
  (void)memspace;
  (void)plist;
  return transfer(dset, filespace, (char *)buf, 0);
}
