// Stand-ins for the few Win32 names the reference uses on its solver path.
#pragma once
#include <climits>
#include <unistd.h>
#include <sys/stat.h>
#ifndef MAX_PATH
#define MAX_PATH 260
#endif
typedef unsigned long DWORD;
#define INVALID_FILE_ATTRIBUTES ((DWORD)-1)
#define FILE_ATTRIBUTE_DIRECTORY 0x10
inline int SetCurrentDirectory(const char*) { return 1; }
inline DWORD GetFileAttributes(const char* p) { struct stat s; if (stat(p, &s) != 0) return INVALID_FILE_ATTRIBUTES; return S_ISDIR(s.st_mode) ? FILE_ATTRIBUTE_DIRECTORY : 0; }
inline DWORD GetLastError() { return 0; }
#define ERROR_ALREADY_EXISTS 183L
#define ERROR_PATH_NOT_FOUND 3L
inline int CreateDirectory(const char* p, void*) { return mkdir(p, 0755) == 0; }
