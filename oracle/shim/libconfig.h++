// Types-only stand-in for the libconfig++ header (TEST INFRASTRUCTURE ONLY).
//
// The reference's graph reader names libconfig only on its "version 4"
// (.cfg) file path. The oracle reads version-2 .bin files exclusively, so
// this stub provides just enough declarations for that code to compile; any
// attempt to actually use it throws.
#ifndef GG_ORACLE_SHIM_LIBCONFIG
#define GG_ORACLE_SHIM_LIBCONFIG
#include <cstdint>
#include <stdexcept>
#include <string>

namespace libconfig {

struct ConfigException : std::runtime_error {
    ConfigException() : std::runtime_error("libconfig stub: not available") {}
};
struct FileIOException : ConfigException {};
struct ParseException : ConfigException {
    const char *getFile() const { return ""; }
    int getLine() const { return 0; }
    const char *getError() const { return "libconfig stub"; }
};

class Setting {
public:
    enum Type { TypeNone, TypeInt, TypeInt64, TypeFloat, TypeString,
                TypeBoolean, TypeGroup, TypeArray, TypeList };
    Setting &add(const char *, Type) { throw ConfigException(); }
    Setting &add(const std::string &, Type) { throw ConfigException(); }
    template <typename T> Setting &operator=(const T &) { throw ConfigException(); }
    const Setting &operator[](const char *) const { throw ConfigException(); }
    Setting &operator[](const char *) { throw ConfigException(); }
    operator long long() const { throw ConfigException(); }
    operator long() const { throw ConfigException(); }
    operator unsigned long() const { throw ConfigException(); }
    operator int() const { throw ConfigException(); }
    operator std::string() const { throw ConfigException(); }
    bool exists(const char *) const { return false; }
};

class Config {
public:
    Setting &getRoot() const { throw ConfigException(); }
    void readFile(const char *) { throw FileIOException(); }
    void readFile(const std::string &) { throw FileIOException(); }
    void writeFile(const char *) { throw FileIOException(); }
    void writeFile(const std::string &) { throw FileIOException(); }
};

} // namespace libconfig
#endif
