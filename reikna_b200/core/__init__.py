from .computation import Computation, ComputationCallable, ComputationParameter
from .signature import Annotation, ArrayMetadata, Parameter, Signature, Type
from .transformation import Transformation, TransformationParameter

__all__ = [
    "Annotation",
    "ArrayMetadata",
    "Computation",
    "ComputationCallable",
    "ComputationParameter",
    "Parameter",
    "Signature",
    "Transformation",
    "TransformationParameter",
    "Type",
]
