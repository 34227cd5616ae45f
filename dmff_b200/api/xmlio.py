"""Force-field XML reader with the reference's ``ffinfo`` layout (dmff/api/xmlio.py:12-113).

``parseXML`` returns {"Operators", "AtomTypes", "Residues", "Forces", "ClassToType"}; each
force is {"meta": <attributes of the force tag>, "node": [{"name": tag, "attrib": {...}}]}.
"""
import xml.etree.ElementTree as ET


class XMLIO:
    def __init__(self):
        self._data = {"Operators": [], "AtomTypes": [], "Residues": [], "Forces": {}}

    def loadXML(self, xml: str):
        root = ET.parse(xml).getroot()
        for child in root:
            if child.tag == "Operators":
                self._data["Operators"].extend(list(child))
            elif child.tag == "AtomTypes":
                self._data["AtomTypes"].extend([a for a in child if a.tag == "Type"])
            elif child.tag == "Residues":
                self._data["Residues"].extend([r for r in child if r.tag == "Residue"])
            elif "Force" in child.tag:
                self._data["Forces"].setdefault(child.tag, []).append(child)

    def parseXML(self):
        ret = {"Operators": {}, "AtomTypes": [], "Residues": [], "Forces": {}, "ClassToType": {}}
        for op in self._data["Operators"]:
            ret["Operators"][op.tag] = [{"name": c.tag, "attrib": dict(c.attrib)} for c in op]
        for at in self._data["AtomTypes"]:
            d = dict(at.attrib)
            d.setdefault("element", None)
            ret["AtomTypes"].append(d)
            if "name" in d and "class" in d:
                ret["ClassToType"].setdefault(d["class"], []).append(d["name"])
        for residue in self._data["Residues"]:
            res = {"name": residue.attrib["name"], "particles": [], "bonds": [], "externals": [], "vsites": []}
            for item in residue:
                if item.tag == "Atom":
                    res["particles"].append({k: (v if k in ("name", "type") else float(v))
                                             for k, v in item.attrib.items()})
                elif item.tag == "Bond":
                    res["bonds"].append(dict(item.attrib))
                elif item.tag == "ExternalBond":
                    res["externals"].append(item.attrib["atomName"])
                elif item.tag == "VirtualSite":
                    res["vsites"].append(dict(item.attrib))
            ret["Residues"].append(res)
        for force, nodes in self._data["Forces"].items():
            f = {"meta": dict(nodes[0].attrib), "node": []}
            for node in nodes:
                for child in node:
                    f["node"].append({"name": child.tag, "attrib": dict(child.attrib)})
            ret["Forces"][force] = f
        return ret
