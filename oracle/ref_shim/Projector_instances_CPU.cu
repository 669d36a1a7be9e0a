// Projector_instances_CPU.cu (host shim) -- TEST INFRASTRUCTURE ONLY. The reference's
// Siddon file includes this name last for its explicit instantiations; ref_siddon.cpp
// instantiates the one class it needs itself.
