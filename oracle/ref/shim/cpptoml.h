// Test-infrastructure shim for cpptoml (third-party header-only TOML library;
// the reference's submodule code/ext/cpptoml is empty, commit unknown).
// Implements the subset of cpptoml's API that the reference's settings.cpp and
// the Problem constructors call (settings.cpp:22-323, euler2d.cpp:6-15):
//   parse_file(path), parser{istream}.parse(), table::get_table,
//   table::get_as<T>, table::get_array_of<cpptoml::array>,
//   array::get_array_of<T>, option<T>, parse_exception.
// The parser reads the TOML subset used by the reference's input files:
// [section] headers, `key = value` with strings, integers, floats, booleans
// and (nested) single-line arrays, and `#` comments.
#pragma once
#include <cstdint>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

namespace cpptoml {

class parse_exception : public std::runtime_error
{
  public:
    explicit parse_exception( const std::string& m ) : std::runtime_error( m ) {}
};

template <class T> class option
{
  public:
    option() : _has( false ), _v() {}
    option( T v ) : _has( true ), _v( std::move( v ) ) {}
    explicit operator bool() const { return _has; }
    const T& operator*() const { return _v; }
    const T* operator->() const { return &_v; }
    T value_or( const T& d ) const { return _has ? _v : d; }

  private:
    bool _has;
    T _v;
};

struct node;
using node_ptr = std::shared_ptr<node>;
class array;

// One parsed value: scalar (string / int / float / bool), array or table.
struct node {
    enum kind_t { STR, INT, FLT, BOOL, ARR, TAB } kind = STR;
    std::string s;
    int64_t i = 0;
    double f  = 0.0;
    bool b    = false;
    std::vector<node_ptr> items;
    std::map<std::string, node_ptr> keys;
};

namespace detail {
template <class T> bool convert( const node& n, T& out ) {
    if constexpr( std::is_same<T, std::string>::value ) {
        if( n.kind != node::STR ) return false;
        out = n.s;
        return true;
    }
    else if constexpr( std::is_same<T, bool>::value ) {
        if( n.kind != node::BOOL ) return false;
        out = n.b;
        return true;
    }
    else if constexpr( std::is_floating_point<T>::value ) {
        if( n.kind == node::FLT ) {
            out = T( n.f );
            return true;
        }
        if( n.kind == node::INT ) {
            out = T( n.i );
            return true;
        }
        return false;
    }
    else {
        if( n.kind != node::INT ) return false;
        if( std::is_unsigned<T>::value && n.i < 0 ) return false;
        out = T( n.i );
        return true;
    }
}
}    // namespace detail

class array
{
  public:
    explicit array( node_ptr n ) : _n( std::move( n ) ) {}
    template <class T> option<std::vector<T>> get_array_of() const {
        std::vector<T> out;
        for( auto& it : _n->items ) {
            T v;
            if( !detail::convert( *it, v ) ) return {};
            out.push_back( v );
        }
        return option<std::vector<T>>( out );
    }
    size_t size() const { return _n->items.size(); }

  private:
    node_ptr _n;
};

class table
{
  public:
    explicit table( node_ptr n ) : _n( std::move( n ) ) {}
    std::shared_ptr<table> get_table( const std::string& key ) const {
        auto it = _n->keys.find( key );
        if( it == _n->keys.end() || it->second->kind != node::TAB ) return std::make_shared<table>( std::make_shared<node>( empty_table() ) );
        return std::make_shared<table>( it->second );
    }
    template <class T> option<T> get_as( const std::string& key ) const {
        auto it = _n->keys.find( key );
        if( it == _n->keys.end() ) return {};
        T v;
        if( !detail::convert( *it->second, v ) ) return {};
        return option<T>( v );
    }
    template <class T> option<std::vector<std::shared_ptr<T>>> get_array_of( const std::string& key ) const {
        static_assert( std::is_same<T, array>::value, "only arrays of arrays are supported" );
        auto it = _n->keys.find( key );
        if( it == _n->keys.end() || it->second->kind != node::ARR ) return {};
        std::vector<std::shared_ptr<array>> out;
        for( auto& sub : it->second->items ) {
            if( sub->kind != node::ARR ) return {};
            out.push_back( std::make_shared<array>( sub ) );
        }
        return option<std::vector<std::shared_ptr<array>>>( out );
    }
    bool contains( const std::string& key ) const { return _n->keys.count( key ) != 0; }

  private:
    static node empty_table() {
        node n;
        n.kind = node::TAB;
        return n;
    }
    node_ptr _n;
};

class parser
{
  public:
    explicit parser( std::istream& is ) : _is( is ) {}
    std::shared_ptr<table> parse() {
        auto root  = std::make_shared<node>();
        root->kind = node::TAB;
        node* cur  = root.get();
        std::string line;
        unsigned lineNo = 0;
        while( std::getline( _is, line ) ) {
            ++lineNo;
            _p = line.c_str();
            skip_ws();
            if( *_p == '\0' || *_p == '#' ) continue;
            if( *_p == '[' ) {
                ++_p;
                std::string name;
                while( *_p && *_p != ']' ) name += *_p++;
                if( *_p != ']' ) throw parse_exception( "bad table header on line " + std::to_string( lineNo ) );
                auto t  = std::make_shared<node>();
                t->kind = node::TAB;
                root->keys[trim( name )] = t;
                cur                      = t.get();
                continue;
            }
            std::string key;
            while( *_p && *_p != '=' ) key += *_p++;
            if( *_p != '=' ) throw parse_exception( "expected '=' on line " + std::to_string( lineNo ) );
            ++_p;
            cur->keys[trim( key )] = value( lineNo );
        }
        return std::make_shared<table>( root );
    }

  private:
    static std::string trim( const std::string& s ) {
        size_t a = s.find_first_not_of( " \t\r\"" ), b = s.find_last_not_of( " \t\r\"" );
        return a == std::string::npos ? std::string() : s.substr( a, b - a + 1 );
    }
    void skip_ws() {
        while( *_p == ' ' || *_p == '\t' || *_p == '\r' ) ++_p;
    }
    node_ptr value( unsigned lineNo ) {
        skip_ws();
        auto n = std::make_shared<node>();
        if( *_p == '"' ) {
            ++_p;
            n->kind = node::STR;
            while( *_p && *_p != '"' ) n->s += *_p++;
            if( *_p != '"' ) throw parse_exception( "unterminated string on line " + std::to_string( lineNo ) );
            ++_p;
        }
        else if( *_p == '[' ) {
            ++_p;
            n->kind = node::ARR;
            skip_ws();
            while( *_p && *_p != ']' ) {
                n->items.push_back( value( lineNo ) );
                skip_ws();
                if( *_p == ',' ) ++_p;
                skip_ws();
            }
            if( *_p != ']' ) throw parse_exception( "unterminated array on line " + std::to_string( lineNo ) );
            ++_p;
        }
        else if( std::string( _p, 4 ) == "true" || std::string( _p, 5 ) == "false" ) {
            n->kind = node::BOOL;
            n->b    = *_p == 't';
            _p += n->b ? 4 : 5;
        }
        else {
            std::string tok;
            while( *_p && *_p != ',' && *_p != ']' && *_p != '#' && *_p != ' ' && *_p != '\t' && *_p != '\r' ) tok += *_p++;
            if( tok.empty() ) throw parse_exception( "missing value on line " + std::to_string( lineNo ) );
            if( tok.find_first_of( ".eEn" ) != std::string::npos ) {
                n->kind = node::FLT;
                n->f    = std::stod( tok );
            }
            else {
                n->kind = node::INT;
                n->i    = std::stoll( tok );
            }
        }
        return n;
    }
    std::istream& _is;
    const char* _p = nullptr;
};

inline std::shared_ptr<table> parse_file( const std::string& path ) {
    std::ifstream f( path );
    if( !f ) throw parse_exception( "cannot open " + path );
    parser p{f};
    return p.parse();
}

}    // namespace cpptoml
