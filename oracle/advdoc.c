/*
 * Clean-room reader/writer for ADVENTURE_IO "AdvDoc" container files.
 *
 * TEST INFRASTRUCTURE ONLY.  The reference (lib/std/fileio.c) reads its
 * partitioned model files (MODEL/model/advhddm_in_*.adv) and writes its
 * results (MODEL/result/advhddm_out_*.adv) through ADVENTURE_IO, an external
 * library that the reference does not ship.  This file implements the subset
 * of that API the reference calls (declared in refshim/Adv/AdvDocument.h) so
 * the reference's own sources can be built and run as the oracle under
 * oracle/_ref/.
 *
 * On-disk layout, as observed in the reference's sample model files
 * (main/fullwave/MODEL/model/advhddm_in_0.adv), little endian, per document:
 *   "AdvDoc\0"                 7 bytes magic
 *   int64  payload_length      followed by the payload bytes
 *   int64  header_length       followed by the header:
 *     int32 len + bytes        document id
 *     int32 count              number of properties
 *     count x (int32 len + key bytes, int32 len + value bytes)
 * A file is a plain concatenation of documents.
 */
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "refshim/Adv/AdvDocument.h"

typedef struct {
  char *key;
  char *val;
} Prop;

struct AdvDocument {
  char *did;
  Prop *props;
  int nprops;
  unsigned char *payload;
  int64_t plen;
  int64_t pcap;
  AdvDocFile *owner; /* non-NULL for documents being written */
  AdvDocument *next;
};

struct AdvDocFile {
  char *path;
  int writing;
  AdvDocument *first;
  AdvDocument *last;
};

struct AdvDatabox {
  AdvDocFile **files;
  int nfiles;
};

static char *dupn(const void *src, size_t n) {
  char *s = (char *)malloc(n + 1);
  memcpy(s, src, n);
  s[n] = 0;
  return s;
}

static void append_doc(AdvDocFile *f, AdvDocument *d) {
  d->next = NULL;
  if (f->last)
    f->last->next = d;
  else
    f->first = d;
  f->last = d;
}

static int read_file(AdvDocFile *f) {
  FILE *fp = fopen(f->path, "rb");
  if (!fp) return 0;
  fseek(fp, 0, SEEK_END);
  long size = ftell(fp);
  fseek(fp, 0, SEEK_SET);
  unsigned char *buf = (unsigned char *)malloc(size > 0 ? size : 1);
  if ((long)fread(buf, 1, size, fp) != size) {
    fclose(fp);
    free(buf);
    return 0;
  }
  fclose(fp);
  long off = 0;
  while (off + 7 + 8 <= size) {
    if (memcmp(buf + off, "AdvDoc\0", 7) != 0) break;
    off += 7;
    int64_t plen, hlen;
    memcpy(&plen, buf + off, 8);
    off += 8;
    AdvDocument *d = (AdvDocument *)calloc(1, sizeof(AdvDocument));
    d->payload = (unsigned char *)malloc(plen > 0 ? plen : 1);
    memcpy(d->payload, buf + off, plen);
    d->plen = d->pcap = plen;
    off += plen;
    memcpy(&hlen, buf + off, 8);
    off += 8;
    const unsigned char *h = buf + off;
    int64_t p = 0;
    int32_t len;
    memcpy(&len, h + p, 4);
    p += 4;
    d->did = dupn(h + p, len);
    p += len;
    int32_t cnt;
    memcpy(&cnt, h + p, 4);
    p += 4;
    d->props = (Prop *)calloc(cnt > 0 ? cnt : 1, sizeof(Prop));
    d->nprops = cnt;
    for (int i = 0; i < cnt; i++) {
      memcpy(&len, h + p, 4);
      p += 4;
      d->props[i].key = dupn(h + p, len);
      p += len;
      memcpy(&len, h + p, 4);
      p += 4;
      d->props[i].val = dupn(h + p, len);
      p += len;
    }
    off += hlen;
    append_doc(f, d);
  }
  free(buf);
  return 1;
}

AdvDatabox *adv_dbox_new(void) { return (AdvDatabox *)calloc(1, sizeof(AdvDatabox)); }

adv_bool adv_dbox_add(AdvDatabox *dbox, const char *path) {
  AdvDocFile *f = (AdvDocFile *)calloc(1, sizeof(AdvDocFile));
  f->path = dupn(path, strlen(path));
  if (!read_file(f)) {
    free(f->path);
    free(f);
    return 0;
  }
  dbox->files = (AdvDocFile **)realloc(dbox->files, sizeof(AdvDocFile *) * (dbox->nfiles + 1));
  dbox->files[dbox->nfiles++] = f;
  return 1;
}

static void free_doc(AdvDocument *d) {
  for (int i = 0; i < d->nprops; i++) {
    free(d->props[i].key);
    free(d->props[i].val);
  }
  free(d->props);
  free(d->payload);
  free(d->did);
  free(d);
}

static void free_file(AdvDocFile *f) {
  AdvDocument *d = f->first;
  while (d) {
    AdvDocument *n = d->next;
    free_doc(d);
    d = n;
  }
  free(f->path);
  free(f);
}

void adv_dbox_close(AdvDatabox *dbox) {
  if (!dbox) return;
  for (int i = 0; i < dbox->nfiles; i++) free_file(dbox->files[i]);
  free(dbox->files);
  free(dbox);
}

static const char *prop_get(AdvDocument *d, const char *key) {
  for (int i = 0; i < d->nprops; i++)
    if (strcmp(d->props[i].key, key) == 0) return d->props[i].val;
  return NULL;
}

AdvDocument *adv_dbox_find_by_property(AdvDatabox *dbox, AdvDocument *prev, ...) {
  const char *keys[16], *vals[16];
  int n = 0;
  va_list ap;
  va_start(ap, prev);
  for (;;) {
    const char *k = va_arg(ap, const char *);
    if (!k || n == 16) break;
    keys[n] = k;
    vals[n] = va_arg(ap, const char *);
    n++;
  }
  va_end(ap);
  int passed = (prev == NULL);
  for (int fi = 0; fi < dbox->nfiles; fi++) {
    for (AdvDocument *d = dbox->files[fi]->first; d; d = d->next) {
      if (!passed) {
        if (d == prev) passed = 1;
        continue;
      }
      int ok = 1;
      for (int i = 0; i < n && ok; i++) {
        const char *v = prop_get(d, keys[i]);
        ok = v && vals[i] && strcmp(v, vals[i]) == 0;
      }
      if (ok) return d;
    }
  }
  return NULL;
}

AdvDocFile *adv_dio_file_open(const char *path, const char *mode) {
  AdvDocFile *f = (AdvDocFile *)calloc(1, sizeof(AdvDocFile));
  f->path = dupn(path, strlen(path));
  if (mode && mode[0] == 'c') {
    FILE *fp = fopen(path, "wb");
    if (!fp) {
      free(f->path);
      free(f);
      return NULL;
    }
    fclose(fp);
    f->writing = 1;
  } else if (!read_file(f)) {
    free(f->path);
    free(f);
    return NULL;
  }
  return f;
}

static void put_str(FILE *fp, const char *s) {
  int32_t len = (int32_t)strlen(s);
  fwrite(&len, 4, 1, fp);
  fwrite(s, 1, len, fp);
}

void adv_dio_file_close(AdvDocFile *f) {
  if (!f) return;
  if (f->writing) {
    FILE *fp = fopen(f->path, "wb");
    if (fp) {
      for (AdvDocument *d = f->first; d; d = d->next) {
        fwrite("AdvDoc\0", 1, 7, fp);
        int64_t plen = d->plen;
        fwrite(&plen, 8, 1, fp);
        if (plen) fwrite(d->payload, 1, plen, fp);
        int64_t hlen = 4 + (int64_t)strlen(d->did) + 4;
        for (int i = 0; i < d->nprops; i++)
          hlen += 8 + (int64_t)strlen(d->props[i].key) + (int64_t)strlen(d->props[i].val);
        fwrite(&hlen, 8, 1, fp);
        put_str(fp, d->did);
        int32_t cnt = d->nprops;
        fwrite(&cnt, 4, 1, fp);
        for (int i = 0; i < d->nprops; i++) {
          put_str(fp, d->props[i].key);
          put_str(fp, d->props[i].val);
        }
      }
      fclose(fp);
    }
  }
  free_file(f);
}

AdvDocument *adv_dio_create(AdvDocFile *fp, const char *did) {
  AdvDocument *d = (AdvDocument *)calloc(1, sizeof(AdvDocument));
  d->did = dupn(did, strlen(did));
  d->owner = fp;
  append_doc(fp, d);
  return d;
}

const char *adv_dio_make_documentid(const char *seed) {
  static char buf[1024];
  static unsigned counter = 0;
  counter++;
  snprintf(buf, sizeof(buf), "%08X:%s:%d:%08X", 0x1000u + counter, seed, (int)getpid(), counter * 2654435761u);
  return buf;
}

void adv_dio_close(AdvDocument *doc) { (void)doc; /* documents are owned by their file */ }

const char *adv_dio_get_property(AdvDocument *doc, const char *key) {
  const char *v = prop_get(doc, key);
  return v ? v : "";
}

adv_bool adv_dio_get_property_int32(AdvDocument *doc, const char *key, int32_t *val) {
  const char *v = prop_get(doc, key);
  if (!v) return 0;
  *val = (int32_t)strtol(v, NULL, 10);
  return 1;
}

adv_bool adv_dio_get_property_float64(AdvDocument *doc, const char *key, double *val) {
  const char *v = prop_get(doc, key);
  if (!v) return 0;
  *val = strtod(v, NULL);
  return 1;
}

void adv_dio_set_property(AdvDocument *doc, const char *key, const char *val) {
  for (int i = 0; i < doc->nprops; i++) {
    if (strcmp(doc->props[i].key, key) == 0) {
      free(doc->props[i].val);
      doc->props[i].val = dupn(val, strlen(val));
      return;
    }
  }
  doc->props = (Prop *)realloc(doc->props, sizeof(Prop) * (doc->nprops + 1));
  doc->props[doc->nprops].key = dupn(key, strlen(key));
  doc->props[doc->nprops].val = dupn(val, strlen(val));
  doc->nprops++;
}

void adv_dio_set_property_int32(AdvDocument *doc, const char *key, int32_t val) {
  char buf[64];
  snprintf(buf, sizeof(buf), "%d", (int)val);
  adv_dio_set_property(doc, key, buf);
}

void adv_dio_set_property_float64(AdvDocument *doc, const char *key, double val) {
  char buf[64];
  snprintf(buf, sizeof(buf), "%.17g", val);
  adv_dio_set_property(doc, key, buf);
}

static int rd(AdvDocument *d, adv_off_t off, void *dst, int64_t n) {
  if (off < 0 || off + n > d->plen) {
    memset(dst, 0, n);
    return (int)n;
  }
  memcpy(dst, d->payload + off, n);
  return (int)n;
}

static int wr(AdvDocument *d, adv_off_t off, const void *src, int64_t n) {
  if (off + n > d->pcap) {
    int64_t cap = d->pcap ? d->pcap : 256;
    while (cap < off + n) cap *= 2;
    d->payload = (unsigned char *)realloc(d->payload, cap);
    memset(d->payload + d->pcap, 0, cap - d->pcap);
    d->pcap = cap;
  }
  memcpy(d->payload + off, src, n);
  if (off + n > d->plen) d->plen = off + n;
  return (int)n;
}

int adv_dio_read_int32(AdvDocument *doc, adv_off_t off, int32_t *val) { return rd(doc, off, val, 4); }
int adv_dio_read_int32v(AdvDocument *doc, adv_off_t off, int n, int32_t *val) {
  return rd(doc, off, val, 4 * (int64_t)n);
}
int adv_dio_read_float64(AdvDocument *doc, adv_off_t off, double *val) { return rd(doc, off, val, 8); }
int adv_dio_read_float64v(AdvDocument *doc, adv_off_t off, int n, double *val) {
  return rd(doc, off, val, 8 * (int64_t)n);
}
int adv_dio_write_int32(AdvDocument *doc, adv_off_t off, int32_t val) { return wr(doc, off, &val, 4); }
int adv_dio_write_int32v(AdvDocument *doc, adv_off_t off, int n, const int32_t *val) {
  return wr(doc, off, val, 4 * (int64_t)n);
}
int adv_dio_write_float64(AdvDocument *doc, adv_off_t off, double val) { return wr(doc, off, &val, 8); }
int adv_dio_write_float64v(AdvDocument *doc, adv_off_t off, int n, const double *val) {
  return wr(doc, off, val, 8 * (int64_t)n);
}
