// The oracle instantiates the simple and the weighted gradient loops.
template void RefIter3D::Init1_SG(Volume_CPU<float>*, Sinogram3D_CPU<float>*);
template void RefIter3D::Init2_SG(Volume_CPU<float>*, Volume_CPU<float>*, Sinogram3D_CPU<float>*);
template void RefIter3D::Init3_SG(Sinogram3D_CPU<float>*);
template void RefIter3D::doSimpleGradient(Volume_CPU<float>*, Sinogram3D_CPU<float>*, Volume_CPU<float>*);
template void RefIter3D::doWeightedGradient(Volume_CPU<float>*, Sinogram3D_CPU<float>*, Volume_CPU<float>*);
