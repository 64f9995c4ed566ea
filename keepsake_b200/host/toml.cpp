#include "toml.h"

#include <cmath>
#include <cstdlib>
#include <sstream>

namespace ksb
{
namespace toml
{

Value Value::make_table()
{
    Value v;
    v.kind = Kind::Table;
    v.table = std::make_shared<toml::Table>();
    return v;
}

Value Value::make_array()
{
    Value v;
    v.kind = Kind::Array;
    v.array = std::make_shared<toml::Array>();
    return v;
}

double Value::number() const { return kind == Kind::Integer ? (double)integer : real; }

Value clone(const Value &v)
{
    Value c = v;
    if (v.kind == Value::Kind::Array) {
        c.array = std::make_shared<Array>();
        for (const Value &e : *v.array)
            c.array->push_back(clone(e));
    } else if (v.kind == Value::Kind::Table) {
        c.table = std::make_shared<Table>();
        for (const auto &[k, e] : *v.table)
            (*c.table)[k] = clone(e);
    }
    return c;
}

namespace
{

class Parser
{
  public:
    explicit Parser(const std::string &s) : s_(s) {}

    Table run()
    {
        Table root;
        Table *cur = &root;
        while (true) {
            skip_ws_comments_newlines();
            if (eof())
                break;
            if (peek() == '[') {
                bool aot = peek(1) == '[';
                pos_ += aot ? 2 : 1;
                skip_ws();
                std::vector<std::string> path = parse_key_path();
                skip_ws();
                expect(']');
                if (aot)
                    expect(']');
                cur = aot ? open_array_table(root, path) : open_table(root, path);
                end_of_line();
                continue;
            }
            std::vector<std::string> path = parse_key_path();
            skip_ws();
            expect('=');
            skip_ws();
            Value v = parse_value();
            assign(*cur, path, std::move(v));
            end_of_line();
        }
        return root;
    }

  private:
    const std::string &s_;
    size_t pos_ = 0;
    int line_ = 1;

    [[noreturn]] void fail(const std::string &what) const
    {
        throw Error("TOML line " + std::to_string(line_) + ": " + what);
    }
    bool eof() const { return pos_ >= s_.size(); }
    char peek(size_t k = 0) const { return pos_ + k < s_.size() ? s_[pos_ + k] : '\0'; }
    char get()
    {
        char c = s_[pos_++];
        if (c == '\n')
            ++line_;
        return c;
    }
    void expect(char c)
    {
        if (eof() || peek() != c)
            fail(std::string("expected '") + c + "'");
        get();
    }
    void skip_ws()
    {
        while (!eof() && (peek() == ' ' || peek() == '\t'))
            get();
    }
    void skip_comment()
    {
        if (peek() == '#')
            while (!eof() && peek() != '\n')
                get();
    }
    void skip_ws_comments_newlines()
    {
        while (!eof()) {
            skip_ws();
            skip_comment();
            if (peek() == '\n' || peek() == '\r')
                get();
            else
                break;
        }
    }
    void end_of_line()
    {
        skip_ws();
        skip_comment();
        if (eof())
            return;
        if (peek() == '\r')
            get();
        if (eof())
            return;
        if (peek() != '\n')
            fail("unexpected characters after a value");
        get();
    }

    static bool bare_key_char(char c)
    {
        return (c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z') || (c >= '0' && c <= '9') || c == '_' || c == '-';
    }

    std::string parse_simple_key()
    {
        if (peek() == '"')
            return parse_basic_string();
        if (peek() == '\'')
            return parse_literal_string();
        std::string k;
        while (!eof() && bare_key_char(peek()))
            k += get();
        if (k.empty())
            fail("expected a key");
        return k;
    }

    std::vector<std::string> parse_key_path()
    {
        std::vector<std::string> path{parse_simple_key()};
        while (true) {
            skip_ws();
            if (peek() != '.')
                break;
            get();
            skip_ws();
            path.push_back(parse_simple_key());
        }
        return path;
    }

    std::string parse_basic_string()
    {
        expect('"');
        if (peek() == '"' && peek(1) == '"')
            fail("multi-line strings are not supported");
        std::string out;
        while (true) {
            if (eof() || peek() == '\n')
                fail("unterminated string");
            char c = get();
            if (c == '"')
                break;
            if (c != '\\') {
                out += c;
                continue;
            }
            char e = get();
            switch (e) {
            case 'n': out += '\n'; break;
            case 't': out += '\t'; break;
            case 'r': out += '\r'; break;
            case 'b': out += '\b'; break;
            case 'f': out += '\f'; break;
            case '"': out += '"'; break;
            case '\\': out += '\\'; break;
            case 'u':
            case 'U': {
                int n = e == 'u' ? 4 : 8;
                uint32_t cp = 0;
                for (int k = 0; k < n; ++k) {
                    char h = get();
                    cp <<= 4;
                    if (h >= '0' && h <= '9')
                        cp |= (uint32_t)(h - '0');
                    else if (h >= 'a' && h <= 'f')
                        cp |= (uint32_t)(h - 'a' + 10);
                    else if (h >= 'A' && h <= 'F')
                        cp |= (uint32_t)(h - 'A' + 10);
                    else
                        fail("bad unicode escape");
                }
                // UTF-8 encode
                if (cp < 0x80) {
                    out += (char)cp;
                } else if (cp < 0x800) {
                    out += (char)(0xC0 | (cp >> 6));
                    out += (char)(0x80 | (cp & 0x3F));
                } else if (cp < 0x10000) {
                    out += (char)(0xE0 | (cp >> 12));
                    out += (char)(0x80 | ((cp >> 6) & 0x3F));
                    out += (char)(0x80 | (cp & 0x3F));
                } else {
                    out += (char)(0xF0 | (cp >> 18));
                    out += (char)(0x80 | ((cp >> 12) & 0x3F));
                    out += (char)(0x80 | ((cp >> 6) & 0x3F));
                    out += (char)(0x80 | (cp & 0x3F));
                }
                break;
            }
            default: fail("bad escape sequence");
            }
        }
        return out;
    }

    std::string parse_literal_string()
    {
        expect('\'');
        if (peek() == '\'' && peek(1) == '\'')
            fail("multi-line strings are not supported");
        std::string out;
        while (true) {
            if (eof() || peek() == '\n')
                fail("unterminated string");
            char c = get();
            if (c == '\'')
                break;
            out += c;
        }
        return out;
    }

    Value parse_value()
    {
        Value v;
        char c = peek();
        if (c == '"') {
            v.kind = Value::Kind::String;
            v.str = parse_basic_string();
        } else if (c == '\'') {
            v.kind = Value::Kind::String;
            v.str = parse_literal_string();
        } else if (c == '[') {
            v = parse_array();
        } else if (c == '{') {
            v = parse_inline_table();
        } else if (s_.compare(pos_, 4, "true") == 0 && !bare_key_char(peek(4))) {
            pos_ += 4;
            v.kind = Value::Kind::Boolean;
            v.boolean = true;
        } else if (s_.compare(pos_, 5, "false") == 0 && !bare_key_char(peek(5))) {
            pos_ += 5;
            v.kind = Value::Kind::Boolean;
            v.boolean = false;
        } else {
            v = parse_number();
        }
        return v;
    }

    Value parse_number()
    {
        std::string tok;
        while (!eof()) {
            char c = peek();
            if (bare_key_char(c) || c == '+' || c == '.')
                tok += get();
            else
                break;
        }
        if (tok.empty())
            fail("expected a value");
        std::string t;
        for (char c : tok)
            if (c != '_')
                t += c;
        Value v;
        std::string body = (t[0] == '+' || t[0] == '-') ? t.substr(1) : t;
        bool neg = t[0] == '-';
        if (body == "inf" || body == "nan") {
            v.kind = Value::Kind::Float;
            v.real = body == "inf" ? INFINITY : NAN;
            if (neg)
                v.real = -v.real;
            return v;
        }
        if (body.size() > 2 && body[0] == '0' && (body[1] == 'x' || body[1] == 'o' || body[1] == 'b')) {
            int base = body[1] == 'x' ? 16 : body[1] == 'o' ? 8 : 2;
            char *end = nullptr;
            unsigned long long u = std::strtoull(body.c_str() + 2, &end, base);
            if (*end)
                fail("bad integer '" + tok + "'");
            v.kind = Value::Kind::Integer;
            v.integer = neg ? -(int64_t)u : (int64_t)u;
            return v;
        }
        bool is_float = t.find_first_of(".eE") != std::string::npos;
        char *end = nullptr;
        if (is_float) {
            v.kind = Value::Kind::Float;
            v.real = std::strtod(t.c_str(), &end);
        } else {
            v.kind = Value::Kind::Integer;
            v.integer = std::strtoll(t.c_str(), &end, 10);
        }
        if (!end || *end)
            fail("bad number '" + tok + "'");
        return v;
    }

    Value parse_array()
    {
        expect('[');
        Value v = Value::make_array();
        while (true) {
            skip_ws_comments_newlines();
            if (peek() == ']') {
                get();
                break;
            }
            v.array->push_back(parse_value());
            skip_ws_comments_newlines();
            if (peek() == ',') {
                get();
                continue;
            }
            skip_ws_comments_newlines();
            expect(']');
            break;
        }
        return v;
    }

    Value parse_inline_table()
    {
        expect('{');
        Value v = Value::make_table();
        skip_ws();
        if (peek() == '}') {
            get();
            return v;
        }
        while (true) {
            skip_ws();
            std::vector<std::string> path = parse_key_path();
            skip_ws();
            expect('=');
            skip_ws();
            assign(*v.table, path, parse_value());
            skip_ws();
            if (peek() == ',') {
                get();
                continue;
            }
            expect('}');
            break;
        }
        return v;
    }

    Table *descend(Table &root, const std::vector<std::string> &path, size_t n)
    {
        Table *t = &root;
        for (size_t k = 0; k < n; ++k) {
            Value &v = (*t)[path[k]];
            if (v.kind == Value::Kind::None)
                v = Value::make_table();
            if (v.kind == Value::Kind::Array && !v.array->empty() && v.array->back().kind == Value::Kind::Table) {
                t = v.array->back().table.get();
                continue;
            }
            if (v.kind != Value::Kind::Table)
                fail("key '" + path[k] + "' is not a table");
            t = v.table.get();
        }
        return t;
    }

    void assign(Table &t, const std::vector<std::string> &path, Value v)
    {
        Table *parent = descend(t, path, path.size() - 1);
        Value &slot = (*parent)[path.back()];
        if (slot.kind != Value::Kind::None)
            fail("duplicate key '" + path.back() + "'");
        slot = std::move(v);
    }

    Table *open_table(Table &root, const std::vector<std::string> &path)
    {
        Table *parent = descend(root, path, path.size() - 1);
        Value &slot = (*parent)[path.back()];
        if (slot.kind == Value::Kind::None) {
            slot = Value::make_table();
        } else if (slot.kind != Value::Kind::Table || slot.defined_by_header) {
            fail("table '" + path.back() + "' defined twice");
        }
        slot.defined_by_header = true;
        return slot.table.get();
    }

    Table *open_array_table(Table &root, const std::vector<std::string> &path)
    {
        Table *parent = descend(root, path, path.size() - 1);
        Value &slot = (*parent)[path.back()];
        if (slot.kind == Value::Kind::None)
            slot = Value::make_array();
        if (slot.kind != Value::Kind::Array)
            fail("'" + path.back() + "' is not an array of tables");
        slot.array->push_back(Value::make_table());
        return slot.array->back().table.get();
    }
};

std::string quote(const std::string &s)
{
    std::string o = "\"";
    for (char c : s) {
        if (c == '"' || c == '\\')
            o += '\\';
        if (c == '\n') {
            o += "\\n";
            continue;
        }
        o += c;
    }
    return o + "\"";
}

std::string key_str(const std::string &k)
{
    bool bare = !k.empty();
    for (char c : k)
        if (!((c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z') || (c >= '0' && c <= '9') || c == '_' || c == '-'))
            bare = false;
    return bare ? k : quote(k);
}

void write_value(std::ostringstream &o, const Value &v)
{
    switch (v.kind) {
    case Value::Kind::String: o << quote(v.str); break;
    case Value::Kind::Integer: o << v.integer; break;
    case Value::Kind::Float: {
        if (std::isinf(v.real))
            o << (v.real > 0 ? "inf" : "-inf");
        else if (std::isnan(v.real))
            o << "nan";
        else {
            std::ostringstream t;
            t.precision(17);
            t << v.real;
            std::string s = t.str();
            if (s.find_first_of(".eE") == std::string::npos)
                s += ".0";
            o << s;
        }
        break;
    }
    case Value::Kind::Boolean: o << (v.boolean ? "true" : "false"); break;
    case Value::Kind::Array: {
        o << "[";
        for (size_t i = 0; i < v.array->size(); ++i) {
            if (i)
                o << ", ";
            write_value(o, (*v.array)[i]);
        }
        o << "]";
        break;
    }
    case Value::Kind::Table: {
        o << "{";
        bool first = true;
        for (const auto &[k, e] : *v.table) {
            o << (first ? " " : ", ") << key_str(k) << " = ";
            write_value(o, e);
            first = false;
        }
        o << (first ? "}" : " }");
        break;
    }
    case Value::Kind::None: o << "\"\""; break;
    }
}

} // namespace

Table parse(const std::string &text)
{
    Parser p(text);
    return p.run();
}

std::string write(const Table &t)
{
    std::ostringstream o;
    for (const auto &[k, v] : t) {
        o << key_str(k) << " = ";
        write_value(o, v);
        o << "\n";
    }
    return o.str();
}

} // namespace toml
} // namespace ksb
