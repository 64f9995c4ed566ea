// A TOML subset for the task configuration files: the forms keepsake's configs use.
//   tables [a.b], arrays of tables [[a]], dotted and quoted keys, basic ("...") and literal ('...')
//   strings, integers (with _ separators, hex), floats (exponent, inf, nan), booleans, arrays
//   (nested, multi-line, trailing comma), inline tables, comments.
// Not supported: multi-line strings, dates and times.  Errors throw ksb::toml::Error with the line.
#pragma once
#include <cstdint>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace ksb
{
namespace toml
{

struct Error : std::runtime_error
{
    using std::runtime_error::runtime_error;
};

struct Value;
using Table = std::map<std::string, Value>;
using Array = std::vector<Value>;

struct Value
{
    enum class Kind { None, String, Integer, Float, Boolean, Array, Table };
    Kind kind = Kind::None;
    std::string str;
    int64_t integer = 0;
    double real = 0.0;
    bool boolean = false;
    std::shared_ptr<toml::Array> array;
    std::shared_ptr<toml::Table> table;
    bool defined_by_header = false; // [a.b] tables may be reopened only once

    static Value make_table();
    static Value make_array();
    bool is_number() const { return kind == Kind::Integer || kind == Kind::Float; }
    double number() const; // integer or float
};

// Parses a document; the root is a table.
Table parse(const std::string &text);
// Serialises a table (keys in sorted order; nested tables as inline tables).
std::string write(const Table &t);
// Deep copy (arrays and tables are shared pointers).
Value clone(const Value &v);

} // namespace toml
} // namespace ksb
