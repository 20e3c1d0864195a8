// Minimal stand-in for the FreeImage API used by the reference's film
// (hdrfilm.cpp, saving only). Saving always fails: the oracle harness reads
// the film's data directly and never writes image files.
#pragma once
typedef struct FIBITMAP_ { int unused; } FIBITMAP;
typedef struct { float red, green, blue; } FIRGBF;
typedef int BOOL;
typedef int FREE_IMAGE_FORMAT;
typedef int FREE_IMAGE_TYPE;
enum { FIF_UNKNOWN = -1, FIF_HDR = 26, FIF_EXR = 29 };
enum { FIT_RGBF = 11, FIT_RGBAF = 12 };
#define HDR_DEFAULT 0
#define EXR_DEFAULT 0
typedef void (*FreeImage_OutputMessageFunction)(FREE_IMAGE_FORMAT fif, const char* msg);
inline void FreeImage_SetOutputMessage(FreeImage_OutputMessageFunction) {}
inline const char* FreeImage_GetFormatFromFIF(FREE_IMAGE_FORMAT) { return "unknown"; }
inline FIBITMAP* FreeImage_AllocateT(FREE_IMAGE_TYPE, int, int, int = 8, unsigned = 0, unsigned = 0, unsigned = 0) { return nullptr; }
inline unsigned char* FreeImage_GetScanLine(FIBITMAP*, int) { return nullptr; }
inline BOOL FreeImage_Save(FREE_IMAGE_FORMAT, FIBITMAP*, const char*, int = 0) { return false; }
inline void FreeImage_Unload(FIBITMAP*) {}
