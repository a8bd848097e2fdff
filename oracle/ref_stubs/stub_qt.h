// Minimal Qt stand-ins so the reference library's host sources compile for the
// oracle build.  Only the members the compiled reference files touch exist; the
// IO members do nothing (file output is not part of the checked path).
// Test infrastructure only: nothing in the product links this.
#ifndef DN_ORACLE_STUB_QT_H
#define DN_ORACLE_STUB_QT_H
#include <string>
#include <vector>
#include <list>
#include <map>
#include <set>
#include <cstdio>
#include <ostream>

class QString : public std::string {
public:
  QString() {}
  QString(const char* s) : std::string(s ? s : "") {}
  QString(const std::string& s) : std::string(s) {}
  QString& setNum(long long v) { *this = std::to_string(v); return *this; }
  QString& setNum(unsigned long v) { *this = std::to_string(v); return *this; }
  QString& setNum(int v) { *this = std::to_string(v); return *this; }
  QString& setNum(double v) { *this = std::to_string(v); return *this; }
  QString rightJustified(int n, char c) const {
    std::string s = *this; while ((int)s.size() < n) s = c + s; return QString(s);
  }
  QString operator+(const QString& o) const { return QString(std::string(*this) + std::string(o)); }
  QString operator+(const char* o) const { return QString(std::string(*this) + o); }
  QString right(int n) const { return n >= (int)size() ? *this : QString(substr(size() - n)); }
  QString left(int n) const { return QString(substr(0, n)); }
  const char* toLatin1() const { return c_str(); }
  const char* toAscii() const { return c_str(); }
  std::string toStdString() const { return *this; }
};
inline QString operator+(const char* a, const QString& b) { return QString(std::string(a) + std::string(b)); }
#define qPrintable(s) ((s).c_str())

template <class T> class QVector : public std::vector<T> {
public:
  QVector() {}
  explicit QVector(size_t n) : std::vector<T>(n) {}
  QVector(size_t n, const T& v) : std::vector<T>(n, v) {}
  T& first() { return this->front(); }
  T& last() { return this->back(); }
  const T& at(size_t i) const { return (*this)[i]; }
  void fill(const T& v) { for (auto& x : *this) x = v; }
  void fill(const T& v, size_t n) { this->assign(n, v); }
  QVector& operator<<(const T& v) { this->push_back(v); return *this; }
  void append(const T& v) { this->push_back(v); }
  int count() const { return (int)this->size(); }
  T* data() { return std::vector<T>::data(); }
};
template <class T> class QList : public std::list<T> {
public:
  QList& operator<<(const T& v) { this->push_back(v); return *this; }
  void append(const T& v) { this->push_back(v); }
};
template <class K, class V> class QMap : public std::map<K, V> {};
template <class T> class QSet : public std::set<T> {};

class QIODevice { public: enum OpenMode { ReadOnly = 1, WriteOnly = 2 }; };
class QFile : public QIODevice {
public:
  QFile(const QString&) {}
  QFile(const char*) {}
  bool open(int) { return false; }
  void close() {}
};
class QTextStream {
public:
  QTextStream(QFile*) {}
  template <class T> QTextStream& operator<<(const T&) { return *this; }
  QTextStream& operator<<(std::ostream& (*)(std::ostream&)) { return *this; }
  void setFieldWidth(int) {}
};
class QDataStream {
public:
  enum FloatingPointPrecision { SinglePrecision, DoublePrecision };
  QDataStream() {}
  QDataStream(QFile*) {}
  void setFloatingPointPrecision(FloatingPointPrecision) {}
  template <class T> QDataStream& operator<<(const T&) { return *this; }
  template <class T> QDataStream& operator>>(T&) { return *this; }
};
class QWidget;
template <class K, class V> class QMapIterator {
public:
  QMapIterator(const QMap<K, V>&) {}
  bool hasNext() const { return false; }
  void next() {}
  K key() const { return K(); }
  V value() const { return V(); }
};
class QObject { public: static QString tr(const char* s) { return QString(s); } };
#ifndef foreach
#define foreach(decl, container) for (decl : container)
#endif
#endif
