// Command-line flags with the syntax the reference's binaries accept
// (src/grid/grid.cpp:107-190, src/dft/dft.cpp:88-187): any number of leading
// '-', a case-insensitive name, and "=value"; a flag is present when an
// argument's name part equals it.
#pragma once

#include <cstdlib>
#include <cstring>
#include <string>
#include <strings.h>

namespace cli {

inline const char *name_part(const char *arg, size_t *len)
{
    while (*arg == '-') arg++;
    const char *eq = std::strchr(arg, '=');
    *len = eq ? (size_t)(eq - arg) : std::strlen(arg);
    return arg;
}

inline const char *find(int argc, char **argv, const char *name)
{
    const size_t n = std::strlen(name);
    for (int i = 1; i < argc; i++) {
        size_t len;
        const char *a = name_part(argv[i], &len);
        if (len == n && strncasecmp(a, name, n) == 0) return a;
    }
    return nullptr;
}

inline bool has(int argc, char **argv, const char *name) { return find(argc, argv, name) != nullptr; }

inline bool value(int argc, char **argv, const char *name, std::string *out)
{
    const char *a = find(argc, argv, name);
    if (!a) return false;
    const char *eq = std::strchr(a, '=');
    if (!eq) return false;
    *out = eq + 1;
    return true;
}

inline double number(int argc, char **argv, const char *name, double dflt)
{
    std::string v;
    return value(argc, argv, name, &v) ? std::atof(v.c_str()) : dflt;
}

}  // namespace cli
