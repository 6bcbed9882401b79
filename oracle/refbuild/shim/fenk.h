// fenk.h -- stand-in for the Wageningen "fenk" container/text library that
// SFbox's sources include (Input.h:4, tools.h:3, misc.h:5, sfnewton.h:26).
//
// Test infrastructure only: it lets the oracle build the reference's own
// C++ sources unmodified.  fenk is not vendored with the reference and no
// version is pinned (Makefile:21-27,44 only link -lfenk), so this header
// restates the semantics the reference's code relies on:
//
//   * Text follows SIMULA text semantics: a Text value is a reference to a
//     shared character frame plus (start, length, pos).  Copying a Text copies
//     the reference (both see the same characters; the copy's pos starts at
//     1); Copy() makes a new frame.  *t gives the text's value for comparison;
//     == compares references (every empty text equals notext).
//   * Vector, Matrix and Array<T> are reference counted and shallow: copies
//     and assignments share storage ("only the reference to x is copied",
//     sf_vectoriterations.cpp:101); Dim() gives fresh zero-filled storage.
//     Matrix is stored column-major so &Gi[1][s] addresses a contiguous
//     column over the first index (Lat3D1stO.cpp:209-210).
//   * Infile/Outfile follow SIMULA's image-based files (Inrecord, Inimage,
//     Outtext, Outimage, ...); Head/Link are SIMULA's SIMSET lists.
#ifndef FENK_SHIM_H
#define FENK_SHIM_H

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <climits>
#include <cfloat>
#include <iostream>
#include <fstream>
#include <memory>
#include <string>
#include <vector>
#include <unistd.h>

using namespace std;

typedef bool Boolean;

void fenk_error(const char *what);

// ---------------------------------------------------------------- Text ----
class Text {
  public:
    Text();
    Text(const char *s);
    Text(const std::string &s);
    // a copy refers to the same characters and starts at pos 1: callers that
    // continue a scan take Text& (SF_SegmentBlock.cpp:432), and Input's
    // CheckReal(Text) scans a by-value copy of a value that Getreal already
    // read (Input.cpp:535-541, :876-885)
    Text(const Text &o) : frame_(o.frame_), start_(o.start_), len_(o.len_), pos_(1) {}
    Text &operator=(const Text &o) {
        frame_ = o.frame_;
        start_ = o.start_;
        len_ = o.len_;
        pos_ = 1;
        return *this;
    }
    Text &operator=(const char *s);

    int Length() const { return len_; }
    int Pos() const { return pos_; }
    void Setpos(int i) { pos_ = (i >= 1 && i <= len_ + 1) ? i : len_ + 1; }
    Boolean More() const { return pos_ <= len_; }
    Text &operator--() { if (pos_ > 1) pos_--; return *this; }   // step pos back one character
    char Getchar();
    void Putchar(char c);
    Text Sub(int i, int n) const;
    Text Strip() const;
    Text Frontstrip() const;
    Text Scanto(char c);
    Text Rest() const;
    Text From(int i) const;
    int Getint();
    double Getreal();
    void Putint(int v);
    void Putreal(double v, int n);
    const char *MainC() const;
    std::string str() const;
    std::string operator*() const { return str(); }
    bool SameRef(const Text &o) const;
    char *data() const { return frame_ ? frame_->data() + start_ : nullptr; }

  private:
    std::shared_ptr<std::vector<char>> frame_;
    int start_ = 0, len_ = 0, pos_ = 1;
    mutable std::shared_ptr<std::string> cstr_;
    friend Text Blanks(int);
    friend Text Copy(const Text &);
};

extern const Text notext;
Text Copy(const Text &t);
Text Copy(const char *s);
Text Blanks(int n);
Text operator+(const Text &a, const Text &b);
Text operator+(const Text &a, const char *b);
Text operator+(const char *a, const Text &b);
inline bool operator==(const Text &a, const Text &b) { return a.SameRef(b); }
inline bool operator!=(const Text &a, const Text &b) { return !a.SameRef(b); }
ostream &operator<<(ostream &o, const Text &t);

// ------------------------------------------------------------- files ----
class Infile {
  public:
    Infile() {}
    Infile(const Text &name) : name_(name.str()) {}
    virtual ~Infile();
    Boolean Open(Text image);
    Boolean Close();
    Boolean Endfile() const { return endfile_; }
    void Inimage();
    Boolean Inrecord();
    int Inint();
    double Inreal();
    char Inchar();
    Text Image;
    void attach_stdin() { in_ = stdin; own_ = false; open_ = true; }

  private:
    std::string name_;
    FILE *in_ = nullptr;
    bool own_ = true, open_ = false, endfile_ = true;
    std::string pending_;   // rest of a record longer than the image
    bool have_pending_ = false;
    bool read_line(std::string &line);
    void skip_blanks_to_item();
};

class Outfile {
  public:
    Outfile() {}
    Outfile(const Text &name) : name_(name.str()) {}
    virtual ~Outfile();
    Boolean Open(Text image);
    Boolean Close();
    void Outimage();
    void Breakoutimage();
    void Outtext(const Text &t);
    void Outtext(const char *s) { Outtext(Text(s)); }
    void Outchar(char c);
    void Outint(int v, int w);
    void Outreal(double v, int n, int w);
    void Outfix(double v, int n, int w);
    Text Image;
    void attach_stdout() { out_ = stdout; own_ = false; open_ = true; Image = Blanks(1024); }

  private:
    std::string name_;
    FILE *out_ = nullptr;
    bool own_ = true, open_ = false;
    void put_field(const std::string &s, int w);
};

Outfile &Sysout();
Infile &Sysin();

// ------------------------------------------------------------ Array<T> ----
// Array(n) and Dim(n) index 0..n-1 (SF_ParserBranched.cpp:65-73)
template <class T>
class Array {
  public:
    Array() : lo_(1), hi_(0) {}
    explicit Array(int n) { Dim(0, n - 1); }
    Array(int lo, int hi) { Dim(lo, hi); }
    void Dim(int n) { Dim(0, n - 1); }
    void Dim(int lo, int hi) {
        lo_ = lo;
        hi_ = hi;
        size_t n = hi >= lo ? size_t(hi - lo + 1) : 0;
        data_ = std::shared_ptr<T>(new T[n > 0 ? n : 1](), std::default_delete<T[]>());
    }
    T &operator[](int i) const {
        if (!data_ || i < lo_ || i > hi_) fenk_error("Array index out of range");
        return data_.get()[size_t(i - lo_)];
    }
    int Lowerbound() const { return lo_; }
    int Upperbound() const { return hi_; }

  private:
    std::shared_ptr<T> data_;
    int lo_, hi_;
};

// -------------------------------------------------------------- Vector ----
class Vector {
  public:
    Vector() : lo_(1), hi_(0), p_(nullptr) {}
    Vector(int lo, int hi) { Dim(lo, hi); }
    Vector(double *p, int lo, int hi) : lo_(lo), hi_(hi), p_(p - lo) {}
    void Dim(int lo, int hi);
    double &operator[](int i) const { return p_[i]; }
    int Lowerbound() const { return lo_; }
    int Upperbound() const { return hi_; }
    int Length() const { return hi_ - lo_ + 1; }
    Vector Copy() const;                    // new storage with the same values
    void Copy(const Vector &src);           // values of src into this storage
    double dotproduct(const Vector &o) const;
    double norm() const;
    double *Data() const { return p_ + lo_; }
    Vector &operator+=(const Vector &o);
    Vector &operator-=(const Vector &o);
    Vector &operator*=(double a);
    Vector &operator/=(double a);

  private:
    std::shared_ptr<std::vector<double>> own_;
    int lo_, hi_;
    double *p_;   // element i at p_[i]
};
Vector operator+(const Vector &a, const Vector &b);
Vector operator-(const Vector &a, const Vector &b);
Vector operator*(double a, const Vector &b);
Vector operator*(const Vector &b, double a);
Vector operator/(const Vector &b, double a);
Vector operator-(const Vector &a);
ostream &operator<<(ostream &o, const Vector &v);

// -------------------------------------------------------------- Matrix ----
class Matrix {
  public:
    class Row {
      public:
        Row(double *p, int stride) : p_(p), stride_(stride) {}
        double &operator[](int j) const { return p_[(long long)j * stride_]; }

      private:
        double *p_;
        int stride_;
    };
    Matrix() : IMIN(1), IMAX(0), JMIN(1), JMAX(0), p_(nullptr), rows_(0) {}
    Matrix(int ilo, int ihi, int jlo, int jhi) { Dim(ilo, ihi, jlo, jhi); }
    void Dim(int ilo, int ihi, int jlo, int jhi);
    // element (i, j) at p_[(j - JMIN) * rows + (i - IMIN)]
    Row operator[](int i) const { return Row(p_ + (i - IMIN) - (long long)JMIN * rows_, rows_); }
    int IMIN, IMAX, JMIN, JMAX;

  private:
    std::shared_ptr<std::vector<double>> own_;
    double *p_;
    int rows_;
};

// ---------------------------------------------------------------- Cube ----
class Cube {
  public:
    class Plane {
      public:
        Plane(double *p, int s1, int s2) : p_(p), s1_(s1), s2_(s2) {}
        Matrix::Row operator[](int j) const { return Matrix::Row(p_ + (long long)j * s1_, s2_); }

      private:
        double *p_;
        int s1_, s2_;
    };
    Cube() {}
    Cube(int ilo, int ihi, int jlo, int jhi, int klo, int khi) { Dim(ilo, ihi, jlo, jhi, klo, khi); }
    void Dim(int ilo, int ihi, int jlo, int jhi, int klo, int khi);
    // element (i, j, k) at base + (i-ilo) + (j-jlo)*ni + (k-klo)*ni*nj
    Plane operator[](int i) const {
        return Plane(p_ + (i - ilo_) - (long long)jlo_ * ni_ - (long long)klo_ * ni_ * nj_, ni_, ni_ * nj_);
    }

  private:
    std::shared_ptr<std::vector<double>> own_;
    double *p_ = nullptr;
    int ilo_ = 1, jlo_ = 1, klo_ = 1, ni_ = 0, nj_ = 0;
};

// ---------------------------------------------------------- Head / Link ----
class Head;
class Link {
  public:
    Link() {}
    virtual ~Link();
    void Into(Head &h);
    void Into(Head *h) { Into(*h); }
    void Out();
    Link *Suc() const;
    Link *Pred() const;

  private:
    Head *head_ = nullptr;
    friend class Head;
};

class Head {
  public:
    Head() {}
    ~Head();
    int Cardinal() const { return (int)items_.size(); }
    Boolean Empty() const { return items_.empty(); }
    Link *operator[](int i) const { return (i >= 1 && i <= (int)items_.size()) ? items_[i - 1] : nullptr; }
    Link *First() const { return items_.empty() ? nullptr : items_.front(); }
    Link *Last() const { return items_.empty() ? nullptr : items_.back(); }
    void Clear();

  private:
    std::vector<Link *> items_;
    friend class Link;
};

#endif
