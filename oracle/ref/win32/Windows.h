/*
 * oracle/ref/win32/Windows.h -- TEST INFRASTRUCTURE ONLY.
 *
 * The few Win32 names the reference's asset tools use
 * (platforms/win32_base.h, platforms/win32_bitmap.h), mapped onto stdio
 * and malloc so oracle/build_ref.sh can compile the unmodified tool
 * sources (bmp2texture.cpp) on Linux.  Window calls are no-ops: the tools
 * never open a window.  DWORD is `unsigned long` to match the reference's
 * own declarations of os::readFromFile/os::writeToFile; the BMP header
 * structs use fixed 32-bit fields to keep the on-disk layout.
 */
#pragma once
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>

typedef void *HANDLE, *LPVOID, *HWND;
typedef unsigned long DWORD;
typedef int BOOL;
typedef int32_t LONG;
typedef size_t SIZE_T;
typedef char *LPTSTR;
typedef union { struct { uint32_t LowPart; int32_t HighPart; }; long long QuadPart; } LARGE_INTEGER;
#ifndef FALSE
#define FALSE 0
#define TRUE 1
#endif
#define GENERIC_READ 0x80000000u
#define GENERIC_WRITE 0x40000000u
#define FILE_SHARE_READ 1u
#define OPEN_EXISTING 3u
#define OPEN_ALWAYS 4u
#define FILE_ATTRIBUTE_NORMAL 0x80u
#define FILE_BEGIN 0u
#define MEM_RESERVE 0x2000u
#define MEM_COMMIT 0x1000u
#define PAGE_READWRITE 4u
#define INVALID_HANDLE_VALUE ((HANDLE)(intptr_t)-1)

#pragma pack(push, 2)
typedef struct { uint16_t bfType; uint32_t bfSize; uint16_t bfReserved1, bfReserved2; uint32_t bfOffBits; } BITMAPFILEHEADER;
#pragma pack(pop)
typedef struct {
    uint32_t biSize; int32_t biWidth, biHeight; uint16_t biPlanes, biBitCount;
    uint32_t biCompression, biSizeImage; int32_t biXPelsPerMeter, biYPelsPerMeter; uint32_t biClrUsed, biClrImportant;
} BITMAPINFOHEADER;

inline HANDLE CreateFileA(const char *path, DWORD access, DWORD, void *, DWORD disposition, DWORD, void *) {
    FILE *f = nullptr;
    if (access & GENERIC_WRITE) {
        f = fopen(path, "r+b");                        // OPEN_ALWAYS: an existing file is opened, not truncated
        if (!f && disposition == OPEN_ALWAYS) f = fopen(path, "w+b");
    } else {
        f = fopen(path, "rb");
    }
    return f ? (HANDLE)f : INVALID_HANDLE_VALUE;
}
inline BOOL ReadFile(HANDLE h, LPVOID out, DWORD size, DWORD *done, void *) {
    size_t n = fread(out, 1, size, (FILE *)h);
    if (done) *done = (DWORD)n;
    return n == size;
}
inline BOOL WriteFile(HANDLE h, const void *in, DWORD size, DWORD *done, void *) {
    size_t n = fwrite(in, 1, size, (FILE *)h);
    if (done) *done = (DWORD)n;
    return n == size;
}
inline BOOL CloseHandle(HANDLE h) { return h && h != INVALID_HANDLE_VALUE && fclose((FILE *)h) == 0; }
inline DWORD SetFilePointer(HANDLE h, LONG offset, LONG *, DWORD) {
    return fseek((FILE *)h, offset, SEEK_SET) == 0 ? (DWORD)offset : (DWORD)-1;
}
inline LPVOID VirtualAlloc(LPVOID, SIZE_T size, DWORD, DWORD) { return calloc(1, size); }
inline BOOL QueryPerformanceCounter(LARGE_INTEGER *c) { c->QuadPart = 0; return TRUE; }
inline BOOL SetWindowTextA(HWND, const char *) { return TRUE; }
inline int ShowCursor(BOOL) { return 0; }
inline HWND SetCapture(HWND) { return nullptr; }
inline BOOL ReleaseCapture() { return TRUE; }
