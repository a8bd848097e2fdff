// Minimal VTK stand-ins for the oracle build of the reference sources.  Every
// object accepts the calls the reference's VTK output code makes and does
// nothing; no file is written.  Test infrastructure only.
#ifndef DN_ORACLE_STUB_VTK_H
#define DN_ORACLE_STUB_VTK_H
#include <cstddef>
typedef long long vtkIdType;
#define VTK_HEXAHEDRON 12
#define VTK_TRIANGLE 5
#define VTK_QUAD 9
#define VTK_POLYGON 7
#define VTK_TETRA 10
#define VTK_WEDGE 13
#define VTK_PYRAMID 14

struct vtkStubObject {
  template <class... A> void SetInputData(A...) {}
  template <class... A> void SetFileName(A...) {}
  template <class... A> void SetDataModeToAscii(A...) {}
  template <class... A> void SetDataModeToBinary(A...) {}
  template <class... A> void Write(A...) {}
  template <class... A> void Update(A...) {}
  template <class... A> void SetDimensions(A...) {}
  template <class... A> void InsertNextPoint(A...) {}
  template <class... A> void SetPoints(A...) {}
  template <class... A> void SetName(A...) {}
  template <class... A> void SetNumberOfValues(A...) {}
  template <class... A> void SetNumberOfComponents(A...) {}
  template <class... A> void SetNumberOfTuples(A...) {}
  template <class... A> void SetValue(A...) {}
  template <class... A> void SetTuple(A...) {}
  template <class... A> void SetNumberOfPoints(A...) {}
  template <class... A> void SetPoint(A...) {}
  template <class... A> void Allocate(A...) {}
  template <class... A> void InsertNextCell(A...) {}
  template <class... A> void SetNumberOfBlocks(A...) {}
  template <class... A> void SetBlock(A...) {}
  template <class... A> void AddArray(A...) {}
  template <class... A> void SetXCoordinates(A...) {}
  template <class... A> void SetYCoordinates(A...) {}
  template <class... A> void SetZCoordinates(A...) {}
  template <class... A> void InsertNextValue(A...) {}
  vtkStubObject* GetCellData() { return this; }
  vtkStubObject* GetPointData() { return this; }
  vtkStubObject* GetPoints() { return this; }
  vtkStubObject* GetOutput() { return this; }
  vtkIdType GetNumberOfPoints() { return 0; }
  vtkIdType GetNumberOfCells() { return 0; }
  void GetPoint(vtkIdType, double* x) { x[0] = x[1] = x[2] = 0; }
  void Delete() {}
};
template <class T> class vtkSmartPointer {
  T* m_P;
public:
  vtkSmartPointer() : m_P(nullptr) {}
  vtkSmartPointer(T* p) : m_P(p) {}
  template <class U> vtkSmartPointer(const vtkSmartPointer<U>& o) : m_P((T*)o.GetPointer()) {}
  static vtkSmartPointer<T> New() { return vtkSmartPointer<T>(new T()); }
  T* operator->() const { return m_P; }
  T* GetPointer() const { return m_P; }
  operator T*() const { return m_P; }
};
#define DN_VTK_STUB_CLASS(name) \
  struct name : public vtkStubObject { static name* New() { return new name(); } };
DN_VTK_STUB_CLASS(vtkDataSet)
DN_VTK_STUB_CLASS(vtkUnstructuredGrid)
DN_VTK_STUB_CLASS(vtkStructuredGrid)
DN_VTK_STUB_CLASS(vtkRectilinearGrid)
DN_VTK_STUB_CLASS(vtkPolyData)
DN_VTK_STUB_CLASS(vtkPoints)
DN_VTK_STUB_CLASS(vtkFloatArray)
DN_VTK_STUB_CLASS(vtkCellData)
DN_VTK_STUB_CLASS(vtkMultiBlockDataSet)
DN_VTK_STUB_CLASS(vtkXMLUnstructuredGridWriter)
DN_VTK_STUB_CLASS(vtkXMLMultiBlockDataWriter)
DN_VTK_STUB_CLASS(vtkXMLRectilinearGridWriter)
DN_VTK_STUB_CLASS(vtkSTLReader)
DN_VTK_STUB_CLASS(vtkPLYReader)
#endif
