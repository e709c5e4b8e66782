// Inert VTK stand-ins (see vtkPointData.h).
#pragma once
#include <memory>

enum VTKCellType { VTK_TETRA = 10, VTK_HEXAHEDRON = 12, VTK_QUADRATIC_TETRA = 24, VTK_QUADRATIC_HEXAHEDRON = 25 };

template <class T>
class vtkSmartPointer {
public:
    static vtkSmartPointer New() { vtkSmartPointer s; s.p = std::make_shared<T>(); return s; }
    T* operator->() const { return p.get(); }
    std::shared_ptr<T> p;
};

class vtkPoints {
public:
    void InsertNextPoint(const double*) { }
};
class vtkIdList {
public:
    void InsertNextId(long long) { }
};
class vtkUnstructuredGrid {
public:
    template <class P> void SetPoints(const P&) { }
    template <class L> void InsertNextCell(VTKCellType, const L&) { }
};
class vtkUnstructuredGridWriter {
public:
    void SetFileName(const char*) { }
    template <class D> void SetInputData(const D&) { }
    void Write() { }
};
