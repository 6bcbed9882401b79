// fenk_shim.cpp -- implementation of the fenk stand-in (see fenk.h).
// Test infrastructure for the oracle's build of the reference sources.
#include "fenk.h"

#include <algorithm>
#include <execinfo.h>

void fenk_error(const char *what) {
    fprintf(stderr, "fenk shim: %s\n", what);
    void *frames[32];
    int n = backtrace(frames, 32);
    backtrace_symbols_fd(frames, n, 2);
    fflush(stderr);
    abort();
}

// ---------------------------------------------------------------- Text ----
const Text notext;

Text::Text() {}

Text::Text(const char *s) {
    size_t n = s ? strlen(s) : 0;
    if (n) {
        frame_ = std::make_shared<std::vector<char>>(s, s + n);
        len_ = (int)n;
    }
}

Text::Text(const std::string &s) {
    if (!s.empty()) {
        frame_ = std::make_shared<std::vector<char>>(s.begin(), s.end());
        len_ = (int)s.size();
    }
}

Text &Text::operator=(const char *s) {
    *this = Text(s);
    return *this;
}

std::string Text::str() const { return len_ ? std::string(frame_->data() + start_, (size_t)len_) : std::string(); }

const char *Text::MainC() const {
    cstr_ = std::make_shared<std::string>(str());
    return cstr_->c_str();
}

bool Text::SameRef(const Text &o) const {
    if (len_ == 0 && o.len_ == 0) return true;
    return frame_ == o.frame_ && start_ == o.start_ && len_ == o.len_;
}

char Text::Getchar() {
    if (pos_ > len_) fenk_error("Getchar beyond the end of a text");
    return (*frame_)[start_ + (pos_++) - 1];
}

void Text::Putchar(char c) {
    if (pos_ > len_) fenk_error("Putchar beyond the end of a text");
    (*frame_)[start_ + (pos_++) - 1] = c;
}

Text Text::Sub(int i, int n) const {
    if (n == 0) return notext;
    if (i < 1 || n < 0 || i + n - 1 > len_) fenk_error("Sub out of range");
    Text t;
    t.frame_ = frame_;
    t.start_ = start_ + i - 1;
    t.len_ = n;
    t.pos_ = 1;
    return t;
}

Text Text::Strip() const {
    int n = len_;
    while (n > 0 && (*frame_)[start_ + n - 1] == ' ') n--;
    return Sub(1, n);
}

Text Text::Frontstrip() const {
    int i = 1;
    while (i <= len_ && (*frame_)[start_ + i - 1] == ' ') i++;
    return Sub(i, len_ - i + 1);
}

Text Text::Scanto(char c) {
    int k = pos_;
    while (k <= len_ && (*frame_)[start_ + k - 1] != c) k++;
    Text t = Sub(pos_, k - pos_);
    pos_ = (k <= len_) ? k + 1 : len_ + 1;
    return t;
}

Text Text::Rest() const { return Sub(pos_, len_ - pos_ + 1); }

Text Text::From(int i) const { return Sub(i, len_ - i + 1); }

// integer item from pos: blanks, optional sign, digits, optional exponent
// e/E[+]digits (Input::CheckInt accepts "1e3"); pos moves past the item
int Text::Getint() {
    int k = pos_;
    while (k <= len_ && (*frame_)[start_ + k - 1] == ' ') k++;
    std::string item;
    if (k <= len_ && ((*frame_)[start_ + k - 1] == '+' || (*frame_)[start_ + k - 1] == '-'))
        item += (*frame_)[start_ + (k++) - 1];
    int nd = 0;
    while (k <= len_ && isdigit((unsigned char)(*frame_)[start_ + k - 1])) {
        item += (*frame_)[start_ + (k++) - 1];
        nd++;
    }
    if (!nd) fenk_error("Getint: no integer item");
    long long v = atoll(item.c_str());
    if (k <= len_ && ((*frame_)[start_ + k - 1] == 'e' || (*frame_)[start_ + k - 1] == 'E')) {
        int k2 = k + 1;
        if (k2 <= len_ && (*frame_)[start_ + k2 - 1] == '+') k2++;
        std::string ex;
        while (k2 <= len_ && isdigit((unsigned char)(*frame_)[start_ + k2 - 1])) ex += (*frame_)[start_ + (k2++) - 1];
        if (!ex.empty()) {
            for (int e = atoi(ex.c_str()); e > 0; e--) v *= 10;
            k = k2;
        }
    }
    pos_ = k;
    return (int)v;
}

double Text::Getreal() {
    int k = pos_;
    while (k <= len_ && (*frame_)[start_ + k - 1] == ' ') k++;
    std::string rest = (k <= len_) ? std::string(frame_->data() + start_ + k - 1, (size_t)(len_ - k + 1)) : "";
    char *end = nullptr;
    double v = strtod(rest.c_str(), &end);
    if (end == rest.c_str()) fenk_error("Getreal: no real item");
    pos_ = k + (int)(end - rest.c_str());
    return v;
}

static void put_right(Text &t, const std::string &s) {
    int n = t.Length();
    char *d = t.data();
    if ((int)s.size() > n) {
        for (int i = 0; i < n; i++) d[i] = '*';
    } else {
        int off = n - (int)s.size();
        for (int i = 0; i < off; i++) d[i] = ' ';
        memcpy(d + off, s.data(), s.size());
    }
    t.Setpos(n + 1);
}

void Text::Putint(int v) { put_right(*this, std::to_string(v)); }

void Text::Putreal(double v, int n) {
    char buf[64];
    snprintf(buf, sizeof buf, "%.*e", std::max(n - 1, 0), v);
    put_right(*this, buf);
}

Text Copy(const Text &t) { return Text(t.str()); }
Text Copy(const char *s) { return Text(s); }

Text Blanks(int n) {
    Text t;
    if (n > 0) {
        t.frame_ = std::make_shared<std::vector<char>>((size_t)n, ' ');
        t.len_ = n;
    }
    return t;
}

Text operator+(const Text &a, const Text &b) { return Text(a.str() + b.str()); }
Text operator+(const Text &a, const char *b) { return Text(a.str() + std::string(b ? b : "")); }
Text operator+(const char *a, const Text &b) { return Text(std::string(a ? a : "") + b.str()); }
ostream &operator<<(ostream &o, const Text &t) { return o << t.str(); }

// ------------------------------------------------------------- files ----
Infile::~Infile() {
    if (in_ && own_) fclose(in_);
}

Boolean Infile::Open(Text image) {
    Image = image;
    if (!own_) return true;
    if (in_) fclose(in_);
    in_ = fopen(name_.c_str(), "r");
    open_ = in_ != nullptr;
    endfile_ = !open_;
    have_pending_ = false;
    Image.Setpos(Image.Length() + 1);
    return open_;
}

Boolean Infile::Close() {
    if (in_ && own_) fclose(in_);
    in_ = nullptr;
    open_ = false;
    endfile_ = true;
    return true;
}

bool Infile::read_line(std::string &line) {
    line.clear();
    if (!in_) return false;
    int c;
    bool any = false;
    while ((c = fgetc(in_)) != EOF) {
        any = true;
        if (c == '\n') break;
        if (c != '\r') line += (char)c;
    }
    return any;
}

Boolean Infile::Inrecord() {
    std::string rec;
    if (have_pending_) {
        rec = pending_;
        have_pending_ = false;
    } else if (!read_line(rec)) {
        endfile_ = true;
        if (Image.Length()) {
            Image.data()[0] = 25;
            Image.Setpos(2);
        }
        return false;
    }
    int n = Image.Length();
    if ((int)rec.size() > n) {
        memcpy(Image.data(), rec.data(), (size_t)n);
        pending_ = rec.substr((size_t)n);
        have_pending_ = true;
        Image.Setpos(n + 1);
        return true;
    }
    if (!rec.empty()) memcpy(Image.data(), rec.data(), rec.size());
    Image.Setpos((int)rec.size() + 1);
    return false;
}

void Infile::Inimage() {
    std::string rec;
    int n = Image.Length();
    for (int i = 0; i < n; i++) Image.data()[i] = ' ';
    if (!read_line(rec)) {
        endfile_ = true;
        if (n) Image.data()[0] = 25;
        Image.Setpos(1);
        return;
    }
    memcpy(Image.data(), rec.data(), std::min(rec.size(), (size_t)n));
    Image.Setpos(1);
}

void Infile::skip_blanks_to_item() {
    for (;;) {
        while (Image.More()) {
            char c = Image.Getchar();
            if (c != ' ' && c != '\t') {
                --Image;
                return;
            }
        }
        if (endfile_) fenk_error("Inint/Inreal beyond the end of a file");
        Inimage();
    }
}

int Infile::Inint() {
    skip_blanks_to_item();
    return Image.Getint();
}

double Infile::Inreal() {
    skip_blanks_to_item();
    return Image.Getreal();
}

char Infile::Inchar() {
    if (!Image.More()) Inimage();
    return Image.Getchar();
}

Outfile::~Outfile() {
    if (out_ && own_) fclose(out_);
}

Boolean Outfile::Open(Text image) {
    Image = image;
    Image.Setpos(1);
    if (!own_) return true;
    out_ = fopen(name_.c_str(), "w");
    open_ = out_ != nullptr;
    return open_;
}

Boolean Outfile::Close() {
    if (Image.Pos() > 1) Outimage();
    if (out_ && own_) fclose(out_);
    out_ = nullptr;
    open_ = false;
    return true;
}

void Outfile::Outimage() {
    int n = Image.Pos() - 1;
    int last = Image.Length();
    while (last > 0 && Image.data()[last - 1] == ' ') last--;
    n = std::max(n, last);
    if (out_) {
        if (n > 0) fwrite(Image.data(), 1, (size_t)n, out_);
        fputc('\n', out_);
        if (!own_) fflush(out_);
    }
    for (int i = 0; i < Image.Length(); i++) Image.data()[i] = ' ';
    Image.Setpos(1);
}

void Outfile::Breakoutimage() {
    int n = Image.Pos() - 1;
    if (out_ && n > 0) {
        fwrite(Image.data(), 1, (size_t)n, out_);
        if (!own_) fflush(out_);
    }
    for (int i = 0; i < Image.Length(); i++) Image.data()[i] = ' ';
    Image.Setpos(1);
}

void Outfile::Outchar(char c) {
    if (!Image.More()) Outimage();
    Image.Putchar(c);
}

void Outfile::Outtext(const Text &t) {
    std::string s = t.str();
    int room = Image.Length() - Image.Pos() + 1;
    if ((int)s.size() > room && Image.Pos() > 1) Outimage();
    for (char c : s) Outchar(c);
}

void Outfile::put_field(const std::string &s, int w) {
    std::string f = s;
    if ((int)f.size() < w) f = std::string((size_t)(w - (int)f.size()), ' ') + f;
    int room = Image.Length() - Image.Pos() + 1;
    if ((int)f.size() > room && Image.Pos() > 1) Outimage();
    for (char c : f) Outchar(c);
}

void Outfile::Outint(int v, int w) { put_field(std::to_string(v), w); }

void Outfile::Outreal(double v, int n, int w) {
    char buf[64];
    snprintf(buf, sizeof buf, "%.*e", std::max(n - 1, 0), v);
    put_field(buf, w);
}

void Outfile::Outfix(double v, int n, int w) {
    char buf[64];
    snprintf(buf, sizeof buf, "%.*f", std::max(n, 0), v);
    put_field(buf, w);
}

Outfile &Sysout() {
    static Outfile *o = [] {
        Outfile *f = new Outfile();
        f->attach_stdout();
        return f;
    }();
    return *o;
}

Infile &Sysin() {
    static Infile *i = [] {
        Infile *f = new Infile();
        f->attach_stdin();
        f->Image = Blanks(1024);
        f->Image.Setpos(1025);
        return f;
    }();
    return *i;
}

// -------------------------------------------------------------- Vector ----
void Vector::Dim(int lo, int hi) {
    lo_ = lo;
    hi_ = hi;
    size_t n = hi >= lo ? size_t(hi - lo + 1) : 0;
    own_ = std::make_shared<std::vector<double>>(n > 0 ? n : 1, 0.0);
    p_ = own_->data() - lo;
}

Vector Vector::Copy() const {
    Vector v(lo_, hi_);
    for (int i = lo_; i <= hi_; i++) v[i] = (*this)[i];
    return v;
}

void Vector::Copy(const Vector &src) {
    for (int i = lo_; i <= hi_; i++) (*this)[i] = src[i];
}

double Vector::dotproduct(const Vector &o) const {
    double s = 0;
    for (int i = lo_; i <= hi_; i++) s += (*this)[i] * o[i];
    return s;
}

double Vector::norm() const { return sqrt(dotproduct(*this)); }

Vector &Vector::operator+=(const Vector &o) {
    for (int i = lo_; i <= hi_; i++) (*this)[i] += o[i];
    return *this;
}
Vector &Vector::operator-=(const Vector &o) {
    for (int i = lo_; i <= hi_; i++) (*this)[i] -= o[i];
    return *this;
}
Vector &Vector::operator*=(double a) {
    for (int i = lo_; i <= hi_; i++) (*this)[i] *= a;
    return *this;
}
Vector &Vector::operator/=(double a) {
    for (int i = lo_; i <= hi_; i++) (*this)[i] /= a;
    return *this;
}

Vector operator+(const Vector &a, const Vector &b) {
    Vector v(a.Lowerbound(), a.Upperbound());
    for (int i = a.Lowerbound(); i <= a.Upperbound(); i++) v[i] = a[i] + b[i];
    return v;
}
Vector operator-(const Vector &a, const Vector &b) {
    Vector v(a.Lowerbound(), a.Upperbound());
    for (int i = a.Lowerbound(); i <= a.Upperbound(); i++) v[i] = a[i] - b[i];
    return v;
}
Vector operator*(double a, const Vector &b) {
    Vector v(b.Lowerbound(), b.Upperbound());
    for (int i = b.Lowerbound(); i <= b.Upperbound(); i++) v[i] = a * b[i];
    return v;
}
Vector operator*(const Vector &b, double a) { return a * b; }
Vector operator/(const Vector &b, double a) {
    Vector v(b.Lowerbound(), b.Upperbound());
    for (int i = b.Lowerbound(); i <= b.Upperbound(); i++) v[i] = b[i] / a;
    return v;
}
Vector operator-(const Vector &a) {
    Vector v(a.Lowerbound(), a.Upperbound());
    for (int i = a.Lowerbound(); i <= a.Upperbound(); i++) v[i] = -a[i];
    return v;
}
ostream &operator<<(ostream &o, const Vector &v) {
    for (int i = v.Lowerbound(); i <= v.Upperbound(); i++) o << v[i] << (i < v.Upperbound() ? " " : "");
    return o;
}

// -------------------------------------------------------------- Matrix ----
void Matrix::Dim(int ilo, int ihi, int jlo, int jhi) {
    IMIN = ilo;
    IMAX = ihi;
    JMIN = jlo;
    JMAX = jhi;
    rows_ = ihi >= ilo ? ihi - ilo + 1 : 0;
    size_t cols = jhi >= jlo ? size_t(jhi - jlo + 1) : 0;
    own_ = std::make_shared<std::vector<double>>(std::max<size_t>((size_t)rows_ * cols, 1), 0.0);
    p_ = own_->data();
}

void Cube::Dim(int ilo, int ihi, int jlo, int jhi, int klo, int khi) {
    ilo_ = ilo;
    jlo_ = jlo;
    klo_ = klo;
    ni_ = ihi >= ilo ? ihi - ilo + 1 : 0;
    nj_ = jhi >= jlo ? jhi - jlo + 1 : 0;
    size_t nk = khi >= klo ? size_t(khi - klo + 1) : 0;
    own_ = std::make_shared<std::vector<double>>(std::max<size_t>((size_t)ni_ * nj_ * nk, 1), 0.0);
    p_ = own_->data();
}

// ---------------------------------------------------------- Head / Link ----
Link::~Link() { Out(); }

void Link::Into(Head &h) {
    Out();
    h.items_.push_back(this);
    head_ = &h;
}

void Link::Out() {
    if (!head_) return;
    auto &v = head_->items_;
    v.erase(std::remove(v.begin(), v.end(), this), v.end());
    head_ = nullptr;
}

Link *Link::Suc() const {
    if (!head_) return nullptr;
    auto &v = head_->items_;
    auto it = std::find(v.begin(), v.end(), this);
    return (it != v.end() && it + 1 != v.end()) ? *(it + 1) : nullptr;
}

Link *Link::Pred() const {
    if (!head_) return nullptr;
    auto &v = head_->items_;
    auto it = std::find(v.begin(), v.end(), this);
    return (it != v.end() && it != v.begin()) ? *(it - 1) : nullptr;
}

Head::~Head() { Clear(); }

void Head::Clear() {
    for (Link *l : items_) l->head_ = nullptr;
    items_.clear();
}
