/*
 * Minimal declarations of the ADVENTURE_IO document API ("libdocio") that the
 * reference's file readers and writers call (lib/std/fileio.c, lib/std/iofunc.c).
 *
 * ADVENTURE_IO is an external library that the reference links but does not
 * ship.  This header declares only the calls the reference makes; the
 * implementation lives in oracle/advdoc.c (written from the on-disk layout of
 * the reference's sample model files, not from ADVENTURE_IO's sources).
 *
 * TEST INFRASTRUCTURE ONLY: used to build the reference itself as a CPU
 * oracle under oracle/_ref/.  Nothing in the product links it.
 */
#ifndef FW_ORACLE_ADVDOCUMENT_SHIM_H
#define FW_ORACLE_ADVDOCUMENT_SHIM_H

#include <stdint.h>

typedef struct AdvDocument AdvDocument;
typedef struct AdvDatabox AdvDatabox;
typedef struct AdvDocFile AdvDocFile;
typedef int64_t adv_off_t;
typedef int adv_bool;

/* data box: a set of opened document files searched by property */
AdvDatabox *adv_dbox_new(void);
adv_bool adv_dbox_add(AdvDatabox *dbox, const char *path);
void adv_dbox_close(AdvDatabox *dbox);
/* varargs: key, value, key, value, ..., NULL */
AdvDocument *adv_dbox_find_by_property(AdvDatabox *dbox, AdvDocument *prev, ...);

/* document files */
AdvDocFile *adv_dio_file_open(const char *path, const char *mode);
void adv_dio_file_close(AdvDocFile *fp);
AdvDocument *adv_dio_create(AdvDocFile *fp, const char *did);
const char *adv_dio_make_documentid(const char *seed);
void adv_dio_close(AdvDocument *doc);

/* properties */
const char *adv_dio_get_property(AdvDocument *doc, const char *key);
adv_bool adv_dio_get_property_int32(AdvDocument *doc, const char *key, int32_t *val);
adv_bool adv_dio_get_property_float64(AdvDocument *doc, const char *key, double *val);
void adv_dio_set_property(AdvDocument *doc, const char *key, const char *val);
void adv_dio_set_property_int32(AdvDocument *doc, const char *key, int32_t val);
void adv_dio_set_property_float64(AdvDocument *doc, const char *key, double val);

/* payload i/o; each returns the number of bytes read or written */
int adv_dio_read_int32(AdvDocument *doc, adv_off_t off, int32_t *val);
int adv_dio_read_int32v(AdvDocument *doc, adv_off_t off, int n, int32_t *val);
int adv_dio_read_float64(AdvDocument *doc, adv_off_t off, double *val);
int adv_dio_read_float64v(AdvDocument *doc, adv_off_t off, int n, double *val);
int adv_dio_write_int32(AdvDocument *doc, adv_off_t off, int32_t val);
int adv_dio_write_int32v(AdvDocument *doc, adv_off_t off, int n, const int32_t *val);
int adv_dio_write_float64(AdvDocument *doc, adv_off_t off, double val);
int adv_dio_write_float64v(AdvDocument *doc, adv_off_t off, int n, const double *val);

#endif
