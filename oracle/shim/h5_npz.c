/*
 * The HDF5 reading calls of the reference's C tests (H5Fopen / H5Fclose and the
 * read helpers of src/util.h) served from the .npz fixtures under tests/golden,
 * so that the reference's own test programs (test/*.c, unmodified) build and run
 * without libhdf5.  TEST INFRASTRUCTURE ONLY.
 *
 * H5Fopen maps a fixture path "<dir>/test_<name>_cplx.hdf5" to
 * $RQC_GOLDEN/<name>.npz, "<dir>/test_<name>_real.hdf5" to $RQC_GOLDEN/real/<name>.npz
 * and "<dir>/test_<name>.hdf5" to $RQC_GOLDEN/<name>.npz ($RQC_GOLDEN defaults to
 * tests/golden).  An .npz file is a ZIP archive of .npy arrays stored without
 * compression (numpy.savez); datasets are found through the ZIP central directory
 * and read from their .npy headers (little-endian doubles or integers, C order).
 * Writing is not supported.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "hdf5.h"
#include "util.h"

#define MAXFILES 64
#define MAXENTRIES 256

struct npz_entry
{
	char name[128];
	long data_offset;   /* offset of the .npy payload in the file */
};

struct npz_file
{
	unsigned char* buf;
	long size;
	int nentries;
	struct npz_entry entries[MAXENTRIES];
};

static struct npz_file* files[MAXFILES];

static uint32_t rd16(const unsigned char* p) { return (uint32_t)p[0] | ((uint32_t)p[1] << 8); }
static uint32_t rd32(const unsigned char* p) { return rd16(p) | (rd16(p + 2) << 16); }

static int map_path(const char* path, char* out, size_t n)
{
	const char* base = strrchr(path, '/');
	base = base ? base + 1 : path;
	char name[256];
	snprintf(name, sizeof(name), "%s", base);
	char* dot = strstr(name, ".hdf5");
	if (!dot) return -1;
	*dot = 0;
	const char* stem = strncmp(name, "test_", 5) == 0 ? name + 5 : name;
	const char* dir = getenv("RQC_GOLDEN");
	if (!dir) dir = "tests/golden";
	const size_t len = strlen(stem);
	if (len > 5 && strcmp(stem + len - 5, "_cplx") == 0)
		snprintf(out, n, "%s/%.*s.npz", dir, (int)(len - 5), stem);
	else if (len > 5 && strcmp(stem + len - 5, "_real") == 0)
		snprintf(out, n, "%s/real/%.*s.npz", dir, (int)(len - 5), stem);
	else
		snprintf(out, n, "%s/%s.npz", dir, stem);
	return 0;
}

hid_t H5Fopen(const char* name, unsigned flags, hid_t fapl)
{
	(void)flags;
	(void)fapl;
	char path[512];
	if (map_path(name, path, sizeof(path)) < 0) return -1;
	FILE* fh = fopen(path, "rb");
	if (!fh) return -1;
	fseek(fh, 0, SEEK_END);
	const long size = ftell(fh);
	fseek(fh, 0, SEEK_SET);
	struct npz_file* f = calloc(1, sizeof(*f));
	f->buf = malloc(size > 0 ? size : 1);
	f->size = size;
	if (fread(f->buf, 1, size, fh) != (size_t)size) {
		fclose(fh);
		free(f->buf);
		free(f);
		return -1;
	}
	fclose(fh);
	/* end of central directory record: signature 0x06054b50, no archive comment */
	long eocd = -1;
	for (long p = size - 22; p >= 0 && p >= size - 22 - 65535; p--)
		if (rd32(f->buf + p) == 0x06054b50) { eocd = p; break; }
	if (eocd < 0) { free(f->buf); free(f); return -1; }
	const int count = (int)rd16(f->buf + eocd + 10);
	long cd = (long)rd32(f->buf + eocd + 16);
	for (int k = 0; k < count && f->nentries < MAXENTRIES; k++) {
		if (cd + 46 > size || rd32(f->buf + cd) != 0x02014b50) break;
		const uint32_t namelen = rd16(f->buf + cd + 28), extralen = rd16(f->buf + cd + 30),
		               commentlen = rd16(f->buf + cd + 32);
		const long local = (long)rd32(f->buf + cd + 42);
		struct npz_entry* e = &f->entries[f->nentries++];
		const uint32_t nl = namelen < sizeof(e->name) - 1 ? namelen : (uint32_t)sizeof(e->name) - 1;
		memcpy(e->name, f->buf + cd + 46, nl);
		e->name[nl] = 0;
		/* payload after the local header, its name and its extra field */
		e->data_offset = local + 30 + rd16(f->buf + local + 26) + rd16(f->buf + local + 28);
		cd += 46 + namelen + extralen + commentlen;
	}
	for (int h = 0; h < MAXFILES; h++)
		if (!files[h]) { files[h] = f; return h + 1; }
	free(f->buf);
	free(f);
	return -1;
}

hid_t H5Fcreate(const char* name, unsigned flags, hid_t fcpl, hid_t fapl)
{
	(void)name; (void)flags; (void)fcpl; (void)fapl;
	return -1;
}

herr_t H5Fclose(hid_t file)
{
	if (file < 1 || file > MAXFILES || !files[file - 1]) return -1;
	free(files[file - 1]->buf);
	free(files[file - 1]);
	files[file - 1] = NULL;
	return 0;
}

/* the .npy array `name` of an open file: element type and count, payload pointer */
static const unsigned char* npy_array(hid_t file, const char* name, char* kind, int* itemsize, long* count, int* ndim,
                                      hsize_t* dims)
{
	if (file < 1 || file > MAXFILES || !files[file - 1]) return NULL;
	const struct npz_file* f = files[file - 1];
	char want[160];
	snprintf(want, sizeof(want), "%s.npy", name);
	for (int k = 0; k < f->nentries; k++) {
		if (strcmp(f->entries[k].name, want) != 0) continue;
		const unsigned char* p = f->buf + f->entries[k].data_offset;
		if (memcmp(p, "\x93NUMPY", 6) != 0) return NULL;
		const int major = p[6];
		const long hlen = major == 1 ? (long)rd16(p + 8) : (long)rd32(p + 8);
		const long hstart = major == 1 ? 10 : 12;
		char header[1024];
		const long hl = hlen < (long)sizeof(header) - 1 ? hlen : (long)sizeof(header) - 1;
		memcpy(header, p + hstart, hl);
		header[hl] = 0;
		const char* d = strstr(header, "'descr': '");
		if (!d || strstr(header, "'fortran_order': True")) return NULL;
		d += 10;
		if (d[0] != '<' && d[0] != '|') return NULL;
		*kind = d[1];
		*itemsize = atoi(d + 2);
		const char* s = strstr(header, "'shape': (");
		if (!s) return NULL;
		s += 10;
		*count = 1;
		*ndim = 0;
		while (*s && *s != ')') {
			char* end;
			const long v = strtol(s, &end, 10);
			if (end == s) { s++; continue; }
			if (dims) dims[*ndim] = (hsize_t)v;
			(*ndim)++;
			*count *= v;
			s = end;
		}
		return p + hstart + hlen;
	}
	return NULL;
}

herr_t read_hdf5_dataset(hid_t file, const char* name, hid_t mem_type, void* data)
{
	char kind;
	int itemsize, ndim;
	long count;
	const unsigned char* p = npy_array(file, name, &kind, &itemsize, &count, &ndim, NULL);
	if (!p) {
		fprintf(stderr, "dataset '%s' not found\n", name);
		return -1;
	}
	for (long i = 0; i < count; i++) {
		double v = 0;
		long long iv = 0;
		if (kind == 'f' && itemsize == 8) { memcpy(&v, p + 8 * i, 8); iv = (long long)v; }
		else if (kind == 'i' && itemsize == 4) { int32_t t; memcpy(&t, p + 4 * i, 4); iv = t; v = (double)t; }
		else if (kind == 'i' && itemsize == 8) { int64_t t; memcpy(&t, p + 8 * i, 8); iv = t; v = (double)t; }
		else if (kind == 'b' && itemsize == 1) { iv = p[i]; v = (double)iv; }
		else return -1;
		if (mem_type == H5T_NATIVE_DOUBLE) ((double*)data)[i] = v;
		else if (mem_type == H5T_NATIVE_INT) ((int*)data)[i] = (int)iv;
		else return -1;
	}
	return 0;
}

herr_t read_hdf5_attribute(hid_t file, const char* name, hid_t mem_type, void* data)
{
	return read_hdf5_dataset(file, name, mem_type, data);
}

herr_t get_hdf5_dataset_ndims(hid_t file, const char* name, int* ndims)
{
	char kind;
	int itemsize;
	long count;
	return npy_array(file, name, &kind, &itemsize, &count, ndims, NULL) ? 0 : -1;
}

herr_t get_hdf5_dataset_dims(hid_t file, const char* name, hsize_t* dims)
{
	char kind;
	int itemsize, ndim;
	long count;
	return npy_array(file, name, &kind, &itemsize, &count, &ndim, dims) ? 0 : -1;
}

herr_t write_hdf5_dataset(hid_t file, const char* name, int degree, const hsize_t dims[], hid_t mem_type_store,
                          hid_t mem_type_input, const void* data)
{
	(void)file; (void)name; (void)degree; (void)dims; (void)mem_type_store; (void)mem_type_input; (void)data;
	return -1;
}

herr_t write_hdf5_scalar_attribute(hid_t file, const char* name, hid_t mem_type_store, hid_t mem_type_input,
                                   const void* data)
{
	(void)file; (void)name; (void)mem_type_store; (void)mem_type_input; (void)data;
	return -1;
}
