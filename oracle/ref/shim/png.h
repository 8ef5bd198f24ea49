/* Declarations-only stand-in for libpng (absent here), so that the reference's loaders.h ->
 * store_png.h parses. The PNG writer is never instantiated by the oracle harness.
 * TEST INFRASTRUCTURE ONLY. */
#ifndef IMBART_REF_PNG_SHIM_H
#define IMBART_REF_PNG_SHIM_H
#include <csetjmp>
#include <cstddef>
typedef unsigned char png_byte;
typedef png_byte* png_bytep;
typedef size_t png_size_t;
typedef void* png_voidp;
typedef struct png_struct_def png_struct;
typedef png_struct* png_structp;
typedef png_struct** png_structpp;
typedef struct png_info_def png_info;
typedef png_info* png_infop;
typedef png_info** png_infopp;
typedef void (*png_rw_ptr)(png_structp, png_bytep, png_size_t);
typedef void (*png_flush_ptr)(png_structp);
#define PNG_LIBPNG_VER_STRING "0.0.0-shim"
#define PNG_COLOR_TYPE_RGBA 6
#define PNG_COLOR_TYPE_RGB_ALPHA 6
#define PNG_INTERLACE_NONE 0
#define PNG_COMPRESSION_TYPE_DEFAULT 0
#define PNG_COMPRESSION_TYPE_BASE 0
#define PNG_FILTER_TYPE_DEFAULT 0
#define PNG_FILTER_TYPE_BASE 0
jmp_buf& png_jmpbuf_shim(png_structp);
#define png_jmpbuf(p) png_jmpbuf_shim(p)
png_voidp png_get_io_ptr(png_structp);
png_structp png_create_write_struct(const char*, png_voidp, png_voidp, png_voidp);
png_structp png_create_read_struct(const char*, png_voidp, png_voidp, png_voidp);
png_infop png_create_info_struct(png_structp);
void png_destroy_read_struct(png_structpp, png_infopp, png_infopp);
void png_destroy_write_struct(png_structpp, png_infopp);
void png_set_write_fn(png_structp, png_voidp, png_rw_ptr, png_flush_ptr);
void png_set_IHDR(png_structp, png_infop, unsigned, unsigned, int, int, int, int, int);
void png_write_info(png_structp, png_infop);
void png_write_row(png_structp, png_bytep);
void png_write_end(png_structp, png_infop);
#endif
