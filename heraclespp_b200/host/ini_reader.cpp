// ini_reader.cpp -- see ini_reader.hpp.
#include "ini_reader.hpp"

#include <algorithm>
#include <cctype>
#include <cstdlib>
#include <fstream>
#include <sstream>

namespace hcl::host {

namespace {

std::string lower(std::string s)
{
    std::transform(s.begin(), s.end(), s.begin(), [](unsigned char c) { return (char)std::tolower(c); });
    return s;
}

std::string trim(std::string const& s)
{
    size_t b = 0;
    size_t e = s.size();
    while (b < e && std::isspace((unsigned char)s[b])) {
        ++b;
    }
    while (e > b && std::isspace((unsigned char)s[e - 1])) {
        --e;
    }
    return s.substr(b, e - b);
}

// inline ';' comment: a ';' preceded by whitespace starts a comment
std::string strip_inline_comment(std::string const& s)
{
    for (size_t i = 0; i < s.size(); ++i) {
        if (s[i] == ';' && (i == 0 || std::isspace((unsigned char)s[i - 1]))) {
            return s.substr(0, i);
        }
    }
    return s;
}

} // namespace

INIReader::INIReader(std::string const& filename)
{
    std::ifstream f(filename);
    if (!f) {
        m_error = -1;
        return;
    }
    std::stringstream ss;
    ss << f.rdbuf();
    parse(ss.str());
}

INIReader INIReader::from_string(std::string const& text)
{
    INIReader r;
    r.parse(text);
    return r;
}

std::string INIReader::key(std::string const& section, std::string const& name)
{
    return lower(section) + "=" + lower(name);
}

void INIReader::parse(std::string const& text)
{
    std::istringstream in(text);
    std::string line;
    std::string section;
    int lineno = 0;
    while (std::getline(in, line)) {
        ++lineno;
        if (lineno == 1 && line.size() >= 3 && (unsigned char)line[0] == 0xEF && (unsigned char)line[1] == 0xBB &&
            (unsigned char)line[2] == 0xBF) {
            line = line.substr(3);
        }
        std::string s = trim(line);
        if (s.empty() || s[0] == ';' || s[0] == '#') {
            continue;
        }
        if (s[0] == '[') {
            const size_t close = s.find(']');
            if (close == std::string::npos) {
                if (!m_error) {
                    m_error = lineno;
                }
                continue;
            }
            section = trim(s.substr(1, close - 1));
            continue;
        }
        s = trim(strip_inline_comment(s));
        size_t sep = s.find_first_of("=:");
        if (sep == std::string::npos) {
            if (!m_error) {
                m_error = lineno;
            }
            continue;
        }
        const std::string name = trim(s.substr(0, sep));
        const std::string value = trim(s.substr(sep + 1));
        const std::string k = key(section, name);
        auto it = m_values.find(k);
        if (it != m_values.end()) {
            // inih joins repeated keys with a newline (multi-line values)
            it->second += "\n" + value;
        } else {
            m_values[k] = value;
        }
    }
}

bool INIReader::HasValue(std::string const& section, std::string const& name) const
{
    return m_values.count(key(section, name)) > 0;
}

std::string INIReader::Get(std::string const& section, std::string const& name, std::string const& default_value) const
{
    auto it = m_values.find(key(section, name));
    return it == m_values.end() ? default_value : it->second;
}

long INIReader::GetInteger(std::string const& section, std::string const& name, long default_value) const
{
    const std::string v = Get(section, name, "");
    if (v.empty()) {
        return default_value;
    }
    char* end = nullptr;
    const long n = std::strtol(v.c_str(), &end, 0);
    return end > v.c_str() ? n : default_value;
}

double INIReader::GetReal(std::string const& section, std::string const& name, double default_value) const
{
    const std::string v = Get(section, name, "");
    if (v.empty()) {
        return default_value;
    }
    char* end = nullptr;
    const double n = std::strtod(v.c_str(), &end);
    return end > v.c_str() ? n : default_value;
}

bool INIReader::GetBoolean(std::string const& section, std::string const& name, bool default_value) const
{
    const std::string v = lower(Get(section, name, ""));
    if (v == "true" || v == "yes" || v == "on" || v == "1") {
        return true;
    }
    if (v == "false" || v == "no" || v == "off" || v == "0") {
        return false;
    }
    return default_value;
}

} // namespace hcl::host
