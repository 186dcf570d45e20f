// A TOML subset parser for the reconstruction drivers' config files.
//
// The reference parses its configs with toml++ (include/config.h:46-58),
// which is not available here.  The configs use a small part of TOML, and
// this parser reads that part: comments, [tables], [dotted.tables],
// [[arrays.of.tables]], bare and quoted keys (dotted keys too), basic and
// literal strings, integers (with '_' separators, hex/oct/bin), floats (with
// exponents, inf, nan), booleans, arrays (nested, multi-line, trailing
// commas) and inline tables.  Dates and multi-line strings are rejected with
// a clear error.  Errors carry the file name and line.
#pragma once

#include <cmath>
#include <cstdint>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace lc::toml {

struct Value;
using Table = std::map<std::string, Value>;
using Array = std::vector<Value>;

struct Value {
    enum Kind { NONE, STRING, INT, FLOAT, BOOL, ARRAY, TABLE } kind = NONE;
    std::string s;
    int64_t i = 0;
    double f = 0.0;
    bool b = false;
    std::shared_ptr<Array> arr;
    std::shared_ptr<Table> tbl;
    bool table_array = false;  // an array created by [[...]] headers

    bool is_table() const { return kind == TABLE; }
    bool is_array() const { return kind == ARRAY; }
    bool is_string() const { return kind == STRING; }
    bool is_number() const { return kind == INT || kind == FLOAT; }
    double number() const { return kind == INT ? (double)i : f; }
    static Value table() {
        Value v;
        v.kind = TABLE;
        v.tbl = std::make_shared<Table>();
        return v;
    }
    static Value array() {
        Value v;
        v.kind = ARRAY;
        v.arr = std::make_shared<Array>();
        return v;
    }
};

// Parses TOML text; `name` labels error messages.
Table parse(const std::string &text, const std::string &name = "<config>");
Table parse_file(const std::string &path);

// Lookup helpers: nullptr when a key is missing.
const Value *find(const Table &t, const std::string &key);
const Table *find_table(const Table &t, const std::string &key);

}  // namespace lc::toml
