// ini_reader.hpp -- the .ini reader the driver and Param use.
//
// Same observable behaviour as the inih INIReader the reference links
// (vendor/inih, used by utils/param.cpp:14-73): [section] headers, key = value
// or key : value pairs, ';' and '#' full-line comments, ';' inline comments,
// section and key lookups case-insensitive, values trimmed, defaults returned
// for missing keys; GetInteger accepts decimal/hex, GetReal strtod, and
// GetBoolean true/yes/on/1 and false/no/off/0.
#pragma once

#include <map>
#include <string>

namespace hcl::host {

class INIReader
{
public:
    explicit INIReader(std::string const& filename);
    static INIReader from_string(std::string const& text);

    // 0 on success, -1 when the file cannot be opened, or the first line
    // number with a parse error.
    [[nodiscard]] int ParseError() const { return m_error; }

    [[nodiscard]] std::string Get(std::string const& section, std::string const& name,
                                  std::string const& default_value) const;
    [[nodiscard]] long GetInteger(std::string const& section, std::string const& name, long default_value) const;
    [[nodiscard]] double GetReal(std::string const& section, std::string const& name, double default_value) const;
    [[nodiscard]] bool GetBoolean(std::string const& section, std::string const& name, bool default_value) const;
    [[nodiscard]] bool HasValue(std::string const& section, std::string const& name) const;

private:
    INIReader() = default;
    void parse(std::string const& text);
    static std::string key(std::string const& section, std::string const& name);

    int m_error = 0;
    std::map<std::string, std::string> m_values;
};

} // namespace hcl::host
